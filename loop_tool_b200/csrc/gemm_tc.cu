// Family (c) on the 5th-generation tensor cores: tcgen05.mma (kind::f16,
// BF16 inputs, FP32 accumulation in TMEM) fed by TMA through an mbarrier
// pipeline, persistent over a table of problems (one problem for a single
// contraction, hundreds for a batch of uneven matmuls in one launch).
//
// Operands arrive as dense K-major BF16 matrices A'[M, Kp], B'[N, Kp] made by
// k_pack from the contraction's separable FP32 operand description (so the
// same kernel runs matmul, batched matmul and padded convolution).  The
// split-BF16 modes pack A' = [Ah | Al | Ah (| Al)], B' = [Bh | Bh | Bl (| Bl)]
// along K, so one BF16 GEMM accumulates Ah*Bh + Al*Bh + Ah*Bl (+ Al*Bl).
//
// Chunked accumulation.  The tensor core's FP32 accumulation truncates, so
// its error grows linearly with the number of K steps summed into one TMEM
// accumulator (measured: ~1.9e-5 relative at K = 16384 with BF16-exact
// inputs).  The K loop is therefore cut into chunks of kChunk elements, each
// accumulated from zero in one of two TMEM buffers (256 columns each); drain
// warps read a finished chunk back and add it into FP32 registers with
// round-to-nearest adds while the tensor core fills the other buffer.  The
// split-BF16 correction segments land in their own chunks, so they are never
// truncated against the much larger main product.
//
// Roles (320 threads per CTA, one CTA per SM):
//   warp 0 lane 0 : TMA producer                  warp 0 : TMEM alloc/free
//   warp 1 lane 0 : MMA issuer (4 x K=16 tcgen05.mma per 64-wide k block)
//   warps 2..9    : drain + epilogue; warp w reads TMEM lanes 32*(w%4)..+31
//                   and columns 128*((w-2)/4)..+127 of each 128 x 256 tile
// Every wait is bounded: on timeout a flag is raised for the host
// (LTB_ERR_TIMEOUT) and the CTA winds down without hanging.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include "kernels.h"
#include "tc_api.h"

namespace {

constexpr int BM = 128, BN = 256, BK = 64, STAGES = 4;
constexpr int NT = 320;
constexpr int kChunkBlocks = 8;  // 8 x 64 = 512 K elements per accumulator
constexpr uint32_t TMEM_COLS = 512;
constexpr int A_BYTES = BM * BK * 2;
constexpr int B_BYTES = BN * BK * 2;
constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
constexpr long long kWaitCycles = 4000000000LL;  // ~2 s at 1.9 GHz

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n"
      " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for the phase of parity `parity` to complete.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int* err) {
  if (mbar_try(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try(bar, parity)) {
    if (clock64() - t0 > kWaitCycles || *(volatile int*)err) {
      atomicExch(err, 1);
      return false;
    }
  }
  return true;
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, uint32_t bar,
                                            int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

// K-major, 128-byte-swizzled canonical layout: 8-row x 128-byte atoms
// (1024 B) stacked along M/N, LBO unused (1), SBO = 1024 B, version 1.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | (uint64_t)1 << 16 | (uint64_t)(1024 >> 4) << 32 |
         (uint64_t)1 << 46 | (uint64_t)2 << 61;
}

// kind::f16 instruction descriptor: FP32 accumulator, BF16 A and B, both
// K-major, M = 128, N = 256.
constexpr uint32_t kIdesc =
    (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
      : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, "
      "%28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Tile index -> (problem, m0, n0).  Tiles of a problem run M-fastest so
// consecutive CTAs share the B tile in L2.
__device__ __forceinline__ int find_problem(const LtbTcProblem* __restrict__ P, int np,
                                            int64_t t) {
  int lo = 0, hi = np - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (P[mid].tile_start <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Grouped raster: tiles advance along M in groups of kGroupM row blocks, so
// the ~148 tiles in flight cover a compact 16 x 9 block region whose A and
// B panels stay resident in L2.
constexpr int kGroupM = 16;
__device__ __forceinline__ void tile_coords(const LtbTcProblem& p, int64_t lt, int* m0, int* n0) {
  const int64_t per_group = (int64_t)kGroupM * p.tiles_n;
  const int g = (int)(lt / per_group);
  const int idx = (int)(lt - (int64_t)g * per_group);
  const int gm = p.tiles_m - g * kGroupM < kGroupM ? p.tiles_m - g * kGroupM : kGroupM;
  *m0 = (g * kGroupM + idx % gm) * BM;
  *n0 = (idx / gm) * BN;
}

__global__ void __launch_bounds__(NT, 1)
    k_gemm_tc(const LtbTcProblem* __restrict__ probs, int nprob, int64_t total_tiles,
              float* c_override, int* err, const __grid_constant__ LtbTcProblem single,
              const __grid_constant__ CUtensorMap single_a,
              const __grid_constant__ CUtensorMap single_b) {
  // probs == nullptr: one problem passed by value with its tensor maps as
  // kernel parameters (encoded at launch over per-run scratch)
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* chunk_full = empty + STAGES;     // [2] MMA -> drain
  uint64_t* chunk_empty = chunk_full + 2;    // [2] drain -> MMA
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(chunk_empty + 2);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(smem_u32(&full[s]), 1);
      mbar_init(smem_u32(&empty[s]), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(smem_u32(&chunk_full[b]), 1);
      mbar_init(smem_u32(&chunk_empty[b]), 8 * 32);  // every drain thread
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ------------------------------------------------------------ producer
    uint32_t g = 0;  // k blocks issued by this CTA so far
    bool alive = true;
    for (int64_t t = blockIdx.x; t < total_tiles && alive; t += gridDim.x) {
      const LtbTcProblem& p = probs ? probs[find_problem(probs, nprob, t)] : single;
      const CUtensorMap* ma =
          probs ? static_cast<const CUtensorMap*>(p.map_a) : &single_a;
      const CUtensorMap* mb =
          probs ? static_cast<const CUtensorMap*>(p.map_b) : &single_b;
      int m0, n0;
      tile_coords(p, t - p.tile_start, &m0, &n0);
      const int nk = (int)((p.Kp + BK - 1) / BK);
      for (int kb = 0; kb < nk; ++kb, ++g) {
        const int s = g % STAGES;
        const uint32_t ph = (g / STAGES) & 1u;
        if (!mbar_wait(smem_u32(&empty[s]), ph ^ 1u, err)) {
          alive = false;
          break;
        }
        const uint32_t fb = smem_u32(&full[s]);
        mbar_expect_tx(fb, STAGE_BYTES);
        uint8_t* sa = smem + s * STAGE_BYTES;
        tma_load_2d(smem_u32(sa), ma, fb, kb * BK, m0);
        tma_load_2d(smem_u32(sa + A_BYTES), mb, fb, kb * BK, n0);
      }
    }
  } else if (warp == 1 && lane == 0) {
    // ---------------------------------------------------------- MMA issuer
    uint32_t g = 0, q = 0;  // k blocks consumed, chunks produced
    bool alive = true;
    for (int64_t t = blockIdx.x; t < total_tiles && alive; t += gridDim.x) {
      const LtbTcProblem& p = probs ? probs[find_problem(probs, nprob, t)] : single;
      const int nk = (int)((p.Kp + BK - 1) / BK);
      for (int c0 = 0; c0 < nk && alive; c0 += kChunkBlocks, ++q) {
        const int buf = q & 1;
        if (!mbar_wait(smem_u32(&chunk_empty[buf]), ((q >> 1) & 1u) ^ 1u, err)) {
          alive = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t acc = tmem + (uint32_t)(buf * BN);
        const int c1 = c0 + kChunkBlocks < nk ? c0 + kChunkBlocks : nk;
        for (int kb = c0; kb < c1; ++kb, ++g) {
          const int s = g % STAGES;
          if (!mbar_wait(smem_u32(&full[s]), (g / STAGES) & 1u, err)) {
            alive = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t a0 = smem_u32(smem + s * STAGE_BYTES);
          const uint64_t ad = sw128_desc(a0), bd = sw128_desc(a0 + A_BYTES);
#pragma unroll
          for (int kk = 0; kk < BK / 16; ++kk)  // +32 bytes per K=16 step
            mma_bf16(acc, ad + 2 * kk, bd + 2 * kk, (kb != c0) || (kk != 0));
          mma_commit(smem_u32(&empty[s]));  // stage reusable once these finish
        }
        mma_commit(smem_u32(&chunk_full[buf]));  // chunk complete in TMEM
      }
    }
  } else if (warp >= 2) {
    // ------------------------------------------------------ drain/epilogue
    const int quad = warp & 3;            // TMEM lanes 32*quad .. +31
    const int half = (warp - 2) >> 2;     // columns 128*half .. +127
    uint32_t q = 0;
    bool alive = true;
    for (int64_t t = blockIdx.x; t < total_tiles && alive; t += gridDim.x) {
      const LtbTcProblem& p = probs ? probs[find_problem(probs, nprob, t)] : single;
      int m0, n0;
      tile_coords(p, t - p.tile_start, &m0, &n0);
      const int nk = (int)((p.Kp + BK - 1) / BK);
      float run[128];
#pragma unroll
      for (int i = 0; i < 128; ++i) run[i] = 0.f;
      for (int c0 = 0; c0 < nk; c0 += kChunkBlocks, ++q) {
        const int buf = q & 1;
        const bool ok = mbar_wait(smem_u32(&chunk_full[buf]), (q >> 1) & 1u, err);
        if (!__all_sync(0xffffffffu, ok)) {
          alive = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t base =
            tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(buf * BN + half * 128);
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          uint32_t r[32];
          tmem_ld32(base + (uint32_t)(c * 32), r);
          tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < 32; ++i) run[c * 32 + i] += __uint_as_float(r[i]);
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        mbar_arrive(smem_u32(&chunk_empty[buf]));  // buffer free for the MMA
      }
      if (!alive) break;
      // epilogue: this thread owns row m0 + 32*quad + lane, 128 columns
      const int row = m0 + quad * 32 + lane;
      if (row < p.M) {
        const int64_t rbase = p.crow[row];
        float* dst = (c_override ? c_override : p.c) + rbase;
        const int cbase = n0 + half * 128;
#pragma unroll
        for (int c = 0; c < 128; c += 4) {
          const int j = cbase + c;
          if (p.unit_cols && j + 4 <= p.N && ((rbase + j) & 3) == 0) {
            *reinterpret_cast<float4*>(dst + j) =
                make_float4(run[c], run[c + 1], run[c + 2], run[c + 3]);
          } else {
#pragma unroll
            for (int e = 0; e < 4; ++e)
              if (j + e < p.N) dst[p.unit_cols ? j + e : p.ccol[j + e]] = run[c + e];
          }
        }
      }
    }
  }
  __syncwarp();
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(TMEM_COLS));
}

// ------------------------------------------------------------ packing
// Gathers an operand through its separable description and writes the BF16
// split of every element into nseg K-segments of a K-major matrix: bit s of
// seg_mask selects the hi part (1) or the lo part (0, x - hi rounded to
// BF16) for segment s.
__device__ __forceinline__ float pack_fetch(const LtbGemmOperand& op, int64_t rows, int64_t K,
                                            int64_t r, int64_t k) {
  if (r >= rows || k >= K) return 0.f;
  if (op.dense) return __ldg(op.base + r * op.ld_row + k * op.ld_k);
  for (int g = 0; g < op.nguard; ++g) {
    const int32_t v = op.grow[(int64_t)g * rows + r] + op.gk[(int64_t)g * K + k];
    if (v < 0 || v >= op.gub[g]) return 0.f;
  }
  return __ldg(op.base + op.rowoff[r] + op.koff[k]);
}

__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __float2bfloat16_rn(x);
  lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}

// Operands contiguous along k: 4 consecutive k per thread, 128-bit loads and
// 64-bit stores when the dense layout allows.
__global__ void __launch_bounds__(256)
    k_pack_k(LtbGemmOperand op, int64_t rows, int64_t K, __nv_bfloat16* __restrict__ out,
             int64_t Kp, int nseg, int seg_mask) {
  const int64_t k4n = (K + 3) / 4;
  const bool vec = op.dense && op.ld_k == 1 && (op.ld_row & 3) == 0 &&
                   ((reinterpret_cast<uintptr_t>(op.base) & 15) == 0) && (K & 3) == 0;
  for (int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; w < rows * k4n;
       w += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = w / k4n, k = (w - r * k4n) * 4;
    float x[4];
    if (vec) {
      const float4 t = __ldg(reinterpret_cast<const float4*>(op.base + r * op.ld_row + k));
      x[0] = t.x; x[1] = t.y; x[2] = t.z; x[3] = t.w;
    } else {
#pragma unroll
      for (int e = 0; e < 4; ++e) x[e] = pack_fetch(op, rows, K, r, k + e);
    }
    __nv_bfloat16 hi[4], lo[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) split_bf16(x[e], hi[e], lo[e]);
    __nv_bfloat16* dst = out + r * Kp + k;
    if (k == 0)  // K padding of this row: scratch is reused, keep it zero
      for (int64_t c = nseg * K; c < Kp; ++c) out[r * Kp + c] = __float2bfloat16_rn(0.f);
    for (int s = 0; s < nseg; ++s) {
      const __nv_bfloat16* v = (seg_mask >> s) & 1 ? hi : lo;
      __nv_bfloat16* d = dst + s * K;
      if (vec && ((r * Kp + s * K + k) & 3) == 0) {
        __nv_bfloat162 a, b;
        a.x = v[0]; a.y = v[1]; b.x = v[2]; b.y = v[3];
        uint2 u;
        u.x = *reinterpret_cast<uint32_t*>(&a);
        u.y = *reinterpret_cast<uint32_t*>(&b);
        *reinterpret_cast<uint2*>(d) = u;
      } else {
#pragma unroll
        for (int e = 0; e < 4; ++e)
          if (k + e < K) d[e] = v[e];
      }
    }
  }
}

// Operands contiguous along rows (e.g. B[k, n] feeding B'[n, k]): a 32 x 32
// tile transposed through shared memory, reads coalesced along rows, writes
// coalesced along k.
__global__ void __launch_bounds__(256)
    k_pack_r(LtbGemmOperand op, int64_t rows, int64_t K, __nv_bfloat16* __restrict__ out,
             int64_t Kp, int nseg, int seg_mask) {
  __shared__ float tile[32][33];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
  const int64_t r0 = (int64_t)blockIdx.y * 32, k0 = (int64_t)blockIdx.x * 32;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int a = ty + 8 * q;
    tile[tx][a] = pack_fetch(op, rows, K, r0 + tx, k0 + a);
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int a = ty + 8 * q;
    const int64_t r = r0 + a, k = k0 + tx;
    if (r >= rows || k >= K) continue;
    __nv_bfloat16 hi, lo;
    split_bf16(tile[a][tx], hi, lo);
    __nv_bfloat16* dst = out + r * Kp + k;
    if (k == 0)  // K padding of this row: scratch is reused, keep it zero
      for (int64_t c = nseg * K; c < Kp; ++c) out[r * Kp + c] = __float2bfloat16_rn(0.f);
    for (int s = 0; s < nseg; ++s) dst[s * K] = (seg_mask >> s) & 1 ? hi : lo;
  }
}

// Every operand of a batch in one launch: CTAs stride over the 32 x 32
// tiles of all jobs (job found by binary search on tile_start).
__global__ void __launch_bounds__(256)
    k_pack_grouped(const LtbPackJob* __restrict__ jobs, int njobs, int64_t total_tiles) {
  __shared__ float tile[32][33];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int64_t t = blockIdx.x; t < total_tiles; t += gridDim.x) {
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (jobs[mid].tile_start <= t) lo = mid;
      else hi = mid - 1;
    }
    const LtbPackJob& J = jobs[lo];
    const int64_t lt = t - J.tile_start;
    const int64_t r0 = (lt / J.tiles_k) * 32, k0 = (lt % J.tiles_k) * 32;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int a = ty + 8 * q;
      if (J.k_contig)
        tile[a][tx] = pack_fetch(J.op, J.rows, J.K, r0 + a, k0 + tx);
      else
        tile[tx][a] = pack_fetch(J.op, J.rows, J.K, r0 + tx, k0 + a);
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int a = ty + 8 * q;
      const int64_t r = r0 + a, k = k0 + tx;
      if (r < J.rows && k < J.K) {
        __nv_bfloat16 hi, lo;
        split_bf16(tile[a][tx], hi, lo);
        __nv_bfloat16* row = static_cast<__nv_bfloat16*>(J.out) + r * J.Kp;
        if (k == 0)
          for (int64_t c = J.nseg * J.K; c < J.Kp; ++c) row[c] = __float2bfloat16_rn(0.f);
        for (int s = 0; s < J.nseg; ++s) row[k + s * J.K] = (J.seg_mask >> s) & 1 ? hi : lo;
      }
    }
    __syncthreads();
  }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    cudaDriverEntryPointQueryResult q;
    void* p = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

}  // namespace

cudaError_t ltb_make_tmap(void* map, const void* base, int64_t rows, int64_t Kp, int box_rows) {
  auto fn = encode_fn();
  if (!fn) return cudaErrorNotSupported;
  const cuuint64_t dims[2] = {(cuuint64_t)Kp, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)Kp * 2};
  const cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(reinterpret_cast<CUtensorMap*>(map), CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2,
                  const_cast<void*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

int ltb_tc_tile_m() { return BM; }
int ltb_tc_tile_n() { return BN; }

cudaError_t ltb_launch_pack(const LtbGemmOperand& op, int64_t rows, int64_t K, void* out,
                            int64_t Kp, int nseg, int seg_mask, int k_contig, cudaStream_t st) {
  __nv_bfloat16* o = static_cast<__nv_bfloat16*>(out);
  if (k_contig) {
    const int64_t work = rows * ((K + 3) / 4);
    int64_t blocks = (work + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_pack_k<<<(unsigned)blocks, 256, 0, st>>>(op, rows, K, o, Kp, nseg, seg_mask);
  } else {
    dim3 grid((unsigned)((K + 31) / 32), (unsigned)((rows + 31) / 32));
    if (grid.y > 65535) return cudaErrorInvalidConfiguration;
    k_pack_r<<<grid, 256, 0, st>>>(op, rows, K, o, Kp, nseg, seg_mask);
  }
  return cudaGetLastError();
}

cudaError_t ltb_launch_pack_grouped(const LtbPackJob* d_jobs, int njobs, int64_t total_tiles,
                                    int sms, cudaStream_t st) {
  const int64_t grid = total_tiles < (int64_t)sms * 8 ? total_tiles : (int64_t)sms * 8;
  k_pack_grouped<<<(unsigned)grid, 256, 0, st>>>(d_jobs, njobs, total_tiles);
  return cudaGetLastError();
}

size_t ltb_tc_smem_bytes() { return (size_t)STAGES * STAGE_BYTES + 1024 + 256; }

cudaError_t ltb_launch_gemm_tc(const LtbTcProblem* d_probs, int nprob, int64_t total_tiles,
                               float* c_override, int sms, int* err, cudaStream_t st,
                               const LtbTcProblem* single, const void* map_a, const void* map_b) {
  static bool attr = false;
  const size_t smem = ltb_tc_smem_bytes();
  if (!attr) {
    cudaError_t e =
        cudaFuncSetAttribute(k_gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const int grid = (int)(total_tiles < sms ? total_tiles : sms);
  LtbTcProblem one{};
  CUtensorMap ma{}, mb{};
  if (!d_probs) {
    if (!single || !map_a || !map_b) return cudaErrorInvalidValue;
    one = *single;
    ma = *static_cast<const CUtensorMap*>(map_a);
    mb = *static_cast<const CUtensorMap*>(map_b);
  }
  k_gemm_tc<<<grid, NT, smem, st>>>(d_probs, nprob, total_tiles, c_override, err, one, ma, mb);
  return cudaGetLastError();
}
