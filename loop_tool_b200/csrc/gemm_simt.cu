// Family (c), plain FP32 path: register-blocked CUDA-core GEMM over
// "separable" operands, C[i, j] = sum_k A(i, k) * B(j, k) with
//   A(i, k) = a.base[a.rowoff[i] + a.koff[k]]   (0 if a guard fails)
// so the same kernel serves row-major matmul, transposed operands and padded
// convolution as an implicit GEMM (the im2col gather happens in the tile
// loader, never in HBM).  Every output is one chain over k = 0..K-1 in
// order of separately rounded FP32 multiplies and adds, whatever the tile
// loader's form: the arithmetic of the reference's C path (cpp.cpp:467-471
// compiles with cc -std=c99, which does not contract a*b+c into an FMA), so
// plain FP32 contractions match the reference bit for bit.
//
// CTA tile 128 x 128, 16 k per step, 256 threads with 8 x 8 outputs each
// (rows ty*4 + {0..3} and 64 + ty*4 + {0..3}, likewise columns); both
// operand tiles sit in shared memory k-major ([16][128 + 4]) so a thread
// reads its 8 A and 8 B values of one k as four 16-byte loads, double
// buffered with the next step's global loads held in registers.  Each
// operand is loaded in one of three forms chosen per launch
// (ltb_simt_mode):
//   kGather  any operand: offsets from tables (or computed for a dense
//            operand), guards; one operand row per thread, fixed for the
//            whole K loop (its row offset and guard partials stay in
//            registers), 8 k per step -> a warp reads 32 neighbouring rows
//   kVecK    dense with unit stride along k (row-major A): 16-byte loads of
//            4 consecutive k, two rows per thread
//   kVecR    dense with unit stride along rows (row-major B read by
//            columns): 16-byte loads of 4 consecutive rows, two k per thread
//   kGatherT the gather form of an A operand whose per-k entries (k offset,
//            up to 3 guard partials, 32-bit) fit a shared table (K <= 768)
#include <stdint.h>

#include "kernels.h"

namespace {

constexpr int BM = 128, BK = 16, NT = 256, LDS = BM + 4;
constexpr int kHoistG = 4;  // guards whose row partials are kept in registers
// Gathered operands with 32-bit k offsets, K <= kKtab and at most 3 guards:
// the per-k entries {koff[k], gk[0][k], gk[1][k], gk[2][k]} are copied into
// shared memory once per CTA, so an element costs one broadcast 16-byte
// shared load instead of 1 + nguard global loads with 64-bit indexing.
constexpr int kKtab = 768;

struct Tile {
  float s[2][BK][LDS];
};

// Loader of one operand for one CTA tile (rows row0 .. row0 + 127).  The
// operand's fields are read in place from the launch parameters (constant
// bank for single launches), not copied into registers.
template <int MODE>
struct Loader;

__host__ __device__ __forceinline__ bool ktab_ok(const LtbGemmOperand& op, int64_t K) {
  return op.k32 && K <= kKtab && op.nguard <= 3;
}

// Fills kt[k] = {koff, gk0, gk1, gk2} for k < K (caller synchronises).
__device__ __forceinline__ void ktab_fill(const LtbGemmOperand& op, int64_t K, int4* kt) {
  for (int k = threadIdx.x; k < K; k += NT) {
    int4 e;
    e.x = (int)(op.dense ? k * op.ld_k : op.koff[k]);
    e.y = op.nguard > 0 ? op.gk[k] : 0;
    e.z = op.nguard > 1 ? op.gk[K + k] : 0;
    e.w = op.nguard > 2 ? op.gk[2 * K + k] : 0;
    kt[k] = e;
  }
}

template <>
struct Loader<kSimtGather> {
  const LtbGemmOperand& op;
  const int64_t rows, K, r;  // r: this thread's row
  int64_t off;               // element offset of that row
  int32_t g[kHoistG];        // its guard partials (first kHoistG guards)
  bool ok;
  float v[8];

  __device__ __forceinline__ Loader(const LtbGemmOperand& o, int64_t row0, int64_t rows_,
                                    int64_t K_)
      : op(o), rows(rows_), K(K_), r(row0 + (threadIdx.x & (BM - 1))) {
    ok = r < rows;
    off = 0;
    if (ok) off = op.dense ? r * op.ld_row : op.rowoff[r];
#pragma unroll
    for (int q = 0; q < kHoistG; ++q)
      g[q] = q < op.nguard && ok ? op.grow[(int64_t)q * rows + r] : 0;
  }
  __device__ __forceinline__ float one(int k) const {
    if (!ok || k >= K) return 0.f;
    const int ng = op.nguard;
#pragma unroll
    for (int q = 0; q < kHoistG; ++q)
      if (q < ng && (uint32_t)(g[q] + op.gk[(int64_t)q * K + k]) >= (uint32_t)op.gub[q])
        return 0.f;
    for (int q = kHoistG; q < ng; ++q)
      if ((uint32_t)(op.grow[(int64_t)q * rows + r] + op.gk[(int64_t)q * K + k]) >=
          (uint32_t)op.gub[q])
        return 0.f;
    return __ldg(op.base + off + (op.dense ? k * op.ld_k : op.koff[k]));
  }
  static constexpr bool kAsync = false;
  __device__ __forceinline__ void fetch(int k0, float (*)[LDS]) {
    const int kk0 = threadIdx.x >> 7;
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = one(k0 + kk0 + 2 * q);
  }
  __device__ __forceinline__ void stash(float (*s)[LDS]) const {
    const int c = threadIdx.x & (BM - 1), kk0 = threadIdx.x >> 7;
#pragma unroll
    for (int q = 0; q < 8; ++q) s[kk0 + 2 * q][c] = v[q];
  }
};

// The gather form reading its per-k entries from the shared table kt
// (ktab_ok operands): one broadcast 16-byte load per element.
template <>
struct Loader<kSimtGatherT> {
  const LtbGemmOperand& op;
  const int K;
  const int4* kt;
  int64_t off;  // element offset of this thread's row
  int32_t g[3];
  bool ok;
  static constexpr bool kAsync = true;  // elements go global -> shared by cp.async

  __device__ __forceinline__ Loader(const LtbGemmOperand& o, int64_t row0, int64_t rows,
                                    int64_t K_)
      : op(o), K((int)K_), kt(nullptr) {
    const int64_t r = row0 + (threadIdx.x & (BM - 1));
    ok = r < rows;
    off = 0;
    if (ok) off = op.dense ? r * op.ld_row : op.rowoff[r];
#pragma unroll
    for (int q = 0; q < 3; ++q) g[q] = q < op.nguard && ok ? op.grow[(int64_t)q * rows + r] : 0;
  }
  // element k of this thread's row into s[kk][row]: a 4-byte cp.async, or
  // zeros (source size 0) outside the operand or its guards
  __device__ __forceinline__ void one(int k, float* dst) const {
    bool in = ok && k < K;
    const float* src = op.base;
    if (in) {
      const int4 e = kt[k];
      const int ng = op.nguard;
      in = !((ng > 0 && (uint32_t)(g[0] + e.y) >= (uint32_t)op.gub[0]) ||
             (ng > 1 && (uint32_t)(g[1] + e.z) >= (uint32_t)op.gub[1]) ||
             (ng > 2 && (uint32_t)(g[2] + e.w) >= (uint32_t)op.gub[2]));
      if (in) src = op.base + off + e.x;
    }
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(
                     static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
                 "l"(src), "r"(in ? 4 : 0)
                 : "memory");
  }
  __device__ __forceinline__ void fetch(int k0, float (*s)[LDS]) {
    const int c = threadIdx.x & (BM - 1), kk0 = threadIdx.x >> 7;
#pragma unroll
    for (int q = 0; q < 8; ++q) one(k0 + kk0 + 2 * q, &s[kk0 + 2 * q][c]);
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  __device__ __forceinline__ void stash(float (*)[LDS]) const {}
};

// Waits for this thread's cp.async copies (kAsync loaders).
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;" ::: "memory");
}

template <>
struct Loader<kSimtVecK> {
  const float* p[2];  // row starts of this thread's two rows (null: past the end)
  const int64_t K;
  float4 v[2];

  __device__ __forceinline__ Loader(const LtbGemmOperand& op, int64_t row0, int64_t rows,
                                    int64_t K_)
      : K(K_) {
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int64_t r = row0 + (threadIdx.x >> 2) + 64 * i;
      p[i] = r < rows ? op.base + r * op.ld_row + (threadIdx.x & 3) * 4 : nullptr;
    }
  }
  static constexpr bool kAsync = false;
  __device__ __forceinline__ void fetch(int k0, float (*)[LDS]) {
    const bool kin = k0 + (threadIdx.x & 3) * 4 < K;  // K % 4 == 0: all 4 or none
#pragma unroll
    for (int i = 0; i < 2; ++i)
      v[i] = (p[i] && kin) ? __ldg(reinterpret_cast<const float4*>(p[i] + k0))
                           : make_float4(0.f, 0.f, 0.f, 0.f);
  }
  __device__ __forceinline__ void stash(float (*s)[LDS]) const {
    const int k = (threadIdx.x & 3) * 4, c = threadIdx.x >> 2;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      s[k + 0][c + 64 * i] = v[i].x;
      s[k + 1][c + 64 * i] = v[i].y;
      s[k + 2][c + 64 * i] = v[i].z;
      s[k + 3][c + 64 * i] = v[i].w;
    }
  }
};

template <>
struct Loader<kSimtVecR> {
  const LtbGemmOperand& op;
  const float* p;  // this thread's 4 rows at k = 0 (null: past the end)
  const int64_t K;
  float4 v[2];

  __device__ __forceinline__ Loader(const LtbGemmOperand& o, int64_t row0, int64_t rows,
                                    int64_t K_)
      : op(o), K(K_) {
    const int64_t r = row0 + (threadIdx.x & 31) * 4;  // rows % 4 == 0: all 4 or none
    p = r < rows ? op.base + r : nullptr;
  }
  static constexpr bool kAsync = false;
  __device__ __forceinline__ void fetch(int k0, float (*)[LDS]) {
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int k = k0 + (threadIdx.x >> 5) + 8 * i;
      v[i] = (p && k < K) ? __ldg(reinterpret_cast<const float4*>(p + (int64_t)k * op.ld_k))
                          : make_float4(0.f, 0.f, 0.f, 0.f);
    }
  }
  __device__ __forceinline__ void stash(float (*s)[LDS]) const {
#pragma unroll
    for (int i = 0; i < 2; ++i)
      *reinterpret_cast<float4*>(&s[(threadIdx.x >> 5) + 8 * i][(threadIdx.x & 31) * 4]) = v[i];
  }
};

template <int AM, int BMODE>
__device__ __forceinline__ void gemm_tile(const LtbGemmProblem& p, int64_t i0, int64_t j0) {
  __shared__ __align__(16) Tile ta, tb;
  __shared__ int4 kta[AM == kSimtGatherT ? kKtab : 1];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // warps 4 (rows) x 2 (columns), lanes 4 x 8: a warp's A reads touch 4
  // distinct 16-byte words and its B reads 8
  const int ty = (warp >> 1) * 4 + (lane >> 3), tx = (warp & 1) * 8 + (lane & 7);
  Loader<AM> la(p.a, i0, p.M, p.K);
  Loader<BMODE> lb(p.b, j0, p.N, p.K);
  if constexpr (AM == kSimtGatherT) {
    ktab_fill(p.a, p.K, kta);
    __syncthreads();
    la.kt = kta;
  }
  float acc[8][8];
#pragma unroll
  for (int a = 0; a < 8; ++a)
#pragma unroll
    for (int b = 0; b < 8; ++b) acc[a][b] = 0.f;

  const int nk = (int)((p.K + BK - 1) / BK);  // K <= kSimtMaxK (checked at launch)
  constexpr bool async = Loader<AM>::kAsync || Loader<BMODE>::kAsync;
  la.fetch(0, ta.s[0]);
  lb.fetch(0, tb.s[0]);
  la.stash(ta.s[0]);
  lb.stash(tb.s[0]);
  if constexpr (async) cp_async_wait_all();
  __syncthreads();
  for (int t = 0; t < nk; ++t) {
    const int cur = t & 1;
    if (t + 1 < nk) {  // buffer cur ^ 1 was last read before the previous barrier
      la.fetch((t + 1) * BK, ta.s[cur ^ 1]);
      lb.fetch((t + 1) * BK, tb.s[cur ^ 1]);
    }
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      const float4 a0 = *reinterpret_cast<const float4*>(&ta.s[cur][kk][ty * 4]);
      const float4 a1 = *reinterpret_cast<const float4*>(&ta.s[cur][kk][64 + ty * 4]);
      const float4 b0 = *reinterpret_cast<const float4*>(&tb.s[cur][kk][tx * 4]);
      const float4 b1 = *reinterpret_cast<const float4*>(&tb.s[cur][kk][64 + tx * 4]);
      const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
      const float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
      for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = 0; b < 8; ++b) acc[a][b] = __fadd_rn(acc[a][b], __fmul_rn(av[a], bv[b]));
    }
    if (t + 1 < nk) {
      la.stash(ta.s[cur ^ 1]);
      lb.stash(tb.s[cur ^ 1]);
    }
    if constexpr (async) cp_async_wait_all();
    __syncthreads();
  }

  // epilogue: 16-byte stores where four neighbouring columns are adjacent
  // and aligned in the output, scalar stores otherwise
  int64_t c0[2];
  bool cvec[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int64_t j = j0 + h * 64 + tx * 4;
    c0[h] = j < p.N ? p.ccol[j] : 0;
    cvec[h] = j + 3 < p.N && p.ccol[j + 1] == c0[h] + 1 && p.ccol[j + 2] == c0[h] + 2 &&
              p.ccol[j + 3] == c0[h] + 3;
  }
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const int64_t i = i0 + (a >> 2) * 64 + ty * 4 + (a & 3);
    if (i >= p.M) continue;
    float* row = p.c + p.crow[i];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float* dst = row + c0[h];
      if (cvec[h] && (reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
        *reinterpret_cast<float4*>(dst) =
            make_float4(acc[a][h * 4], acc[a][h * 4 + 1], acc[a][h * 4 + 2], acc[a][h * 4 + 3]);
      } else {
        const int64_t j = j0 + h * 64 + tx * 4;
#pragma unroll
        for (int b = 0; b < 4; ++b)
          if (j + b < p.N) row[p.ccol[j + b]] = acc[a][h * 4 + b];
      }
    }
  }
}

// CTAs per SM the register budget is sized for (launch bounds): two (128
// registers per thread) hide load latency for gathered operands and small
// grouped problems; a single launch of a row-major matmul (16-byte loads on
// both sides) runs faster with one CTA and no register cap (measured:
// 49 vs 44 TFLOP/s at 8192^3, 13.8 vs 11.7 at 1000^3).
template <int AM, int BMODE>
constexpr int simt_min_ctas() {
  return AM == kSimtVecK && BMODE == kSimtVecR ? 1 : 2;
}

template <int AM, int BMODE>
__global__ void __launch_bounds__(NT, (simt_min_ctas<AM, BMODE>()))
    k_gemm_simt(LtbGemmProblem p) {
  gemm_tile<AM, BMODE>(p, (int64_t)blockIdx.y * BM, (int64_t)blockIdx.x * BM);
}

// one CTA per 128 x 128 tile of any problem of the batch
template <int AM, int BMODE>
__global__ void __launch_bounds__(NT, 2)
    k_gemm_simt_grouped(const LtbGemmProblem* __restrict__ probs,
                        const int64_t* __restrict__ tile_start, int nprob) {
  const int64_t t = blockIdx.x;
  int lo = 0, hi = nprob - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tile_start[mid] <= t) lo = mid;
    else hi = mid - 1;
  }
  const LtbGemmProblem p = probs[lo];
  const int64_t lt = t - tile_start[lo];
  const int64_t tn = (p.N + BM - 1) / BM;
  gemm_tile<AM, BMODE>(p, (lt / tn) * BM, (lt % tn) * BM);
}

// ------------------------------------------------------------ 64 x 64 tiles
// Problems with fewer 128 x 128 tiles than SMs: 64 x 64 CTA tiles, 256
// threads with 4 x 4 outputs each (rows ty*4 + {0..3}, columns tx*4 +
// {0..3}), 16 k per step, elements fetched one by one (dense offsets
// computed, others from the tables, guards applied).  Each output is the
// same chain of rounded multiplies and adds over k in order as in the
// 128 x 128 kernel, so both give the same bits.
constexpr int MBM = 64, MLD = MBM + 4;

__device__ __forceinline__ float fetch_one(const LtbGemmOperand& op, int64_t r, int64_t k,
                                           int64_t rows, int64_t K) {
  if (r >= rows || k >= K) return 0.f;
  if (op.dense) return __ldg(op.base + r * op.ld_row + k * op.ld_k);
  for (int g = 0; g < op.nguard; ++g) {
    const int32_t v = op.grow[(int64_t)g * rows + r] + op.gk[(int64_t)g * K + k];
    if ((uint32_t)v >= (uint32_t)op.gub[g]) return 0.f;
  }
  return __ldg(op.base + op.rowoff[r] + op.koff[k]);
}

// 64 rows x 16 k of one operand, 4 elements per thread into s[k][row]:
// lanes along k for a k-contiguous dense operand (a warp reads 8 rows x
// 16 k), along rows otherwise (a warp reads 32 neighbouring rows of one k).
struct MidLoader {
  float v[4];
  __device__ __forceinline__ void fetch(const LtbGemmOperand& op, int64_t row0, int64_t rows,
                                        int64_t K, int k0, bool kfast) {
    const int t = threadIdx.x;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int r = kfast ? t >> 2 : t & 63, k = kfast ? (t & 3) * 4 + q : (t >> 6) + 4 * q;
      v[q] = fetch_one(op, row0 + r, k0 + k, rows, K);
    }
  }
  __device__ __forceinline__ void stash(float (*s)[MLD], bool kfast) const {
    const int t = threadIdx.x;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int r = kfast ? t >> 2 : t & 63, k = kfast ? (t & 3) * 4 + q : (t >> 6) + 4 * q;
      s[k][r] = v[q];
    }
  }
};

__global__ void __launch_bounds__(NT) k_gemm_simt_mid(LtbGemmProblem p) {
  __shared__ __align__(16) float sa[2][BK][MLD], sb[2][BK][MLD];
  const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
  const int64_t i0 = (int64_t)blockIdx.y * MBM, j0 = (int64_t)blockIdx.x * MBM;
  const bool akf = p.a.dense && p.a.ld_k == 1, bkf = p.b.dense && p.b.ld_k == 1;
  MidLoader la, lb;
  float acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.f;
  const int nk = (int)((p.K + BK - 1) / BK);  // K <= kSimtMaxK (checked at launch)
  la.fetch(p.a, i0, p.M, p.K, 0, akf);
  lb.fetch(p.b, j0, p.N, p.K, 0, bkf);
  la.stash(sa[0], akf);
  lb.stash(sb[0], bkf);
  __syncthreads();
  for (int t = 0; t < nk; ++t) {
    const int cur = t & 1;
    if (t + 1 < nk) {
      la.fetch(p.a, i0, p.M, p.K, (t + 1) * BK, akf);
      lb.fetch(p.b, j0, p.N, p.K, (t + 1) * BK, bkf);
    }
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      const float4 a4 = *reinterpret_cast<const float4*>(&sa[cur][kk][ty * 4]);
      const float4 b4 = *reinterpret_cast<const float4*>(&sb[cur][kk][tx * 4]);
      const float av[4] = {a4.x, a4.y, a4.z, a4.w};
      const float bv[4] = {b4.x, b4.y, b4.z, b4.w};
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = __fadd_rn(acc[a][b], __fmul_rn(av[a], bv[b]));
    }
    if (t + 1 < nk) {
      la.stash(sa[cur ^ 1], akf);
      lb.stash(sb[cur ^ 1], bkf);
    }
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int64_t i = i0 + ty * 4 + a;
    if (i >= p.M) continue;
    float* row = p.c + p.crow[i];
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int64_t j = j0 + tx * 4 + b;
      if (j < p.N) row[p.ccol[j]] = acc[a][b];
    }
  }
}

template <int AM, int BMODE>
cudaError_t launch_one(const LtbGemmProblem& p, cudaStream_t st) {
  dim3 grid((unsigned)((p.N + BM - 1) / BM), (unsigned)((p.M + BM - 1) / BM));
  if (grid.y > 65535) return cudaErrorInvalidConfiguration;
  k_gemm_simt<AM, BMODE><<<grid, NT, 0, st>>>(p);
  return cudaGetLastError();
}

template <int AM, int BMODE>
cudaError_t launch_grouped(const LtbGemmProblem* d_probs, const int64_t* d_tile_start, int nprob,
                           int64_t total_tiles, cudaStream_t st) {
  k_gemm_simt_grouped<AM, BMODE><<<(unsigned)total_tiles, NT, 0, st>>>(d_probs, d_tile_start,
                                                                        nprob);
  return cudaGetLastError();
}

template <int AM>
cudaError_t dispatch_b(int bm, const LtbGemmProblem* p, const LtbGemmProblem* d_probs,
                       const int64_t* d_tile_start, int nprob, int64_t tiles, cudaStream_t st) {
  switch (bm) {
    case kSimtVecK:
      return p ? launch_one<AM, kSimtVecK>(*p, st)
               : launch_grouped<AM, kSimtVecK>(d_probs, d_tile_start, nprob, tiles, st);
    case kSimtVecR:
      return p ? launch_one<AM, kSimtVecR>(*p, st)
               : launch_grouped<AM, kSimtVecR>(d_probs, d_tile_start, nprob, tiles, st);
    default:
      return p ? launch_one<AM, kSimtGather>(*p, st)
               : launch_grouped<AM, kSimtGather>(d_probs, d_tile_start, nprob, tiles, st);
  }
}

cudaError_t dispatch(int modes, const LtbGemmProblem* p, const LtbGemmProblem* d_probs,
                     const int64_t* d_tile_start, int nprob, int64_t tiles, cudaStream_t st) {
  const int am = modes & 15, bm = (modes >> 4) & 15;
  switch (am) {
    case kSimtGatherT:
      return dispatch_b<kSimtGatherT>(bm, p, d_probs, d_tile_start, nprob, tiles, st);
    case kSimtVecK:
      return dispatch_b<kSimtVecK>(bm, p, d_probs, d_tile_start, nprob, tiles, st);
    case kSimtVecR:
      return dispatch_b<kSimtVecR>(bm, p, d_probs, d_tile_start, nprob, tiles, st);
    default:
      return dispatch_b<kSimtGather>(bm, p, d_probs, d_tile_start, nprob, tiles, st);
  }
}

}  // namespace

int ltb_simt_mode(const LtbGemmOperand& op, int64_t rows, int64_t K, bool a_side) {
  const int gather = a_side && ktab_ok(op, K) ? kSimtGatherT : kSimtGather;
  if (!op.dense || op.nguard != 0 || (reinterpret_cast<uintptr_t>(op.base) & 15) != 0)
    return gather;
  if (op.ld_k == 1 && op.ld_row % 4 == 0 && K % 4 == 0) return kSimtVecK;
  if (op.ld_row == 1 && op.ld_k % 4 == 0 && rows % 4 == 0) return kSimtVecR;
  return gather;
}

int ltb_simt_tile(const LtbGemmProblem& p, int sms, int tile) {
  if (tile == 64 || tile == 128) return tile;
  const int64_t tiles128 = ((p.M + BM - 1) / BM) * ((p.N + BM - 1) / BM);
  // 64-wide tiles pay scalar element fetches; they win only where 128-wide
  // tiles leave most SMs idle (measured: 512^3 63 vs 69 us, 1000^3 134 vs
  // 118 us)
  return tiles128 * 4 <= sms ? 64 : 128;
}

cudaError_t ltb_launch_gemm_simt(const LtbGemmProblem& p, int sms, cudaStream_t st, int tile) {
  if (p.K > kSimtMaxK) return cudaErrorInvalidValue;
  if (ltb_simt_tile(p, sms, tile) == 64) {
    dim3 grid((unsigned)((p.N + MBM - 1) / MBM), (unsigned)((p.M + MBM - 1) / MBM));
    if (grid.y > 65535) return cudaErrorInvalidConfiguration;
    k_gemm_simt_mid<<<grid, NT, 0, st>>>(p);
    return cudaGetLastError();
  }
  const int modes =
      ltb_simt_mode(p.a, p.M, p.K, true) | ltb_simt_mode(p.b, p.N, p.K, false) << 4;
  return dispatch(modes, &p, nullptr, nullptr, 0, 0, st);
}

cudaError_t ltb_launch_gemm_simt_grouped(const LtbGemmProblem* d_probs,
                                         const int64_t* d_tile_start, int nprob,
                                         int64_t total_tiles, int modes, cudaStream_t st) {
  if (total_tiles > 0x7fffffff) return cudaErrorInvalidConfiguration;
  if (total_tiles == 0) return cudaSuccess;
  return dispatch(modes, nullptr, d_probs, d_tile_start, nprob, total_tiles, st);
}
