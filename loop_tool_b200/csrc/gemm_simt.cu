// Family (c), plain FP32 path: register-blocked CUDA-core GEMM over
// "separable" operands, C[i, j] = sum_k A(i, k) * B(j, k) with
//   A(i, k) = a.base[a.rowoff[i] + a.koff[k]]   (0 if a guard fails)
// so the same kernel serves row-major matmul, transposed operands, batched
// matmul (grid.z) and padded convolution as an implicit GEMM (the im2col
// gather happens in the tile loader, never in HBM).
#include "kernels.h"

namespace {

constexpr int BM = 128, BN = 128, BK = 8, TM = 8, TN = 8, NT = 256;

__device__ __forceinline__ float gather(const LtbGemmOperand& op, int64_t r,
                                        int64_t k, int64_t rows, int64_t K) {
  if (r >= rows || k >= K) return 0.f;
  if (op.dense) return __ldg(op.base + r * op.ld_row + k * op.ld_k);
  for (int g = 0; g < op.nguard; ++g) {
    const int32_t v = op.grow[(int64_t)g * rows + r] + op.gk[(int64_t)g * K + k];
    if (v < 0 || v >= op.gub[g]) return 0.f;
  }
  return __ldg(op.base + op.rowoff[r] + op.koff[k]);
}

__device__ void gemm_tile(const LtbGemmProblem& p, int64_t i0, int64_t j0);

__global__ void __launch_bounds__(NT)
    k_gemm_simt(LtbGemmProblem p) {
  gemm_tile(p, (int64_t)blockIdx.y * BM, (int64_t)blockIdx.x * BN);
}

// one CTA per 128 x 128 tile of any problem of the batch
__global__ void __launch_bounds__(NT)
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
  const int64_t tn = (p.N + BN - 1) / BN;
  gemm_tile(p, (lt / tn) * BM, (lt % tn) * BN);
}

__device__ void gemm_tile(const LtbGemmProblem& p, int64_t i0, int64_t j0) {
  __shared__ float As[2][BK][BM];
  __shared__ float Bs[2][BK][BN];
  const int tid = threadIdx.x;
  // loader mapping: A tile 128 rows x 8 k -> thread loads 4 k of one row
  const int a_r = tid >> 1, a_k = (tid & 1) * 4;
  // B tile 8 k x 128 cols -> thread loads 4 cols of one k
  const int b_k = tid >> 5, b_c = (tid & 31) * 4;
  const int ty = tid >> 4, tx = tid & 15;
  float acc[TM][TN];
#pragma unroll
  for (int a = 0; a < TM; ++a)
#pragma unroll
    for (int b = 0; b < TN; ++b) acc[a][b] = 0.f;

  float ra[4], rb[4];
  auto fetch = [&](int64_t k0) {
#pragma unroll
    for (int q = 0; q < 4; ++q) ra[q] = gather(p.a, i0 + a_r, k0 + a_k + q, p.M, p.K);
#pragma unroll
    for (int q = 0; q < 4; ++q) rb[q] = gather(p.b, j0 + b_c + q, k0 + b_k, p.N, p.K);
  };
  auto stash = [&](int buf) {
#pragma unroll
    for (int q = 0; q < 4; ++q) As[buf][a_k + q][a_r] = ra[q];
    *reinterpret_cast<float4*>(&Bs[buf][b_k][b_c]) = make_float4(rb[0], rb[1], rb[2], rb[3]);
  };
  const int64_t nk = (p.K + BK - 1) / BK;
  fetch(0);
  stash(0);
  __syncthreads();
  for (int64_t t = 0; t < nk; ++t) {
    const int cur = t & 1;
    if (t + 1 < nk) fetch((t + 1) * BK);
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      float av[TM], bv[TN];
      const float4 a0 = *reinterpret_cast<const float4*>(&As[cur][kk][ty * 4]);
      const float4 a1 = *reinterpret_cast<const float4*>(&As[cur][kk][64 + ty * 4]);
      const float4 b0 = *reinterpret_cast<const float4*>(&Bs[cur][kk][tx * 4]);
      const float4 b1 = *reinterpret_cast<const float4*>(&Bs[cur][kk][64 + tx * 4]);
      av[0] = a0.x; av[1] = a0.y; av[2] = a0.z; av[3] = a0.w;
      av[4] = a1.x; av[5] = a1.y; av[6] = a1.z; av[7] = a1.w;
      bv[0] = b0.x; bv[1] = b0.y; bv[2] = b0.z; bv[3] = b0.w;
      bv[4] = b1.x; bv[5] = b1.y; bv[6] = b1.z; bv[7] = b1.w;
#pragma unroll
      for (int a = 0; a < TM; ++a)
#pragma unroll
        for (int b = 0; b < TN; ++b) acc[a][b] = fmaf(av[a], bv[b], acc[a][b]);
    }
    if (t + 1 < nk) stash(cur ^ 1);
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < TM; ++a) {
    const int64_t i = i0 + (a < 4 ? ty * 4 + a : 64 + ty * 4 + (a - 4));
    if (i >= p.M) continue;
    const int64_t rbase = p.crow[i];
#pragma unroll
    for (int b = 0; b < TN; ++b) {
      const int64_t j = j0 + (b < 4 ? tx * 4 + b : 64 + tx * 4 + (b - 4));
      if (j < p.N) p.c[rbase + p.ccol[j]] = acc[a][b];
    }
  }
}

}  // namespace

cudaError_t ltb_launch_gemm_simt(const LtbGemmProblem& p, int sms,
                                 cudaStream_t st) {
  (void)sms;
  dim3 grid((unsigned)((p.N + BN - 1) / BN), (unsigned)((p.M + BM - 1) / BM));
  if (grid.y > 65535) return cudaErrorInvalidConfiguration;
  k_gemm_simt<<<grid, NT, 0, st>>>(p);
  return cudaGetLastError();
}

cudaError_t ltb_launch_gemm_simt_grouped(const LtbGemmProblem* d_probs,
                                         const int64_t* d_tile_start, int nprob,
                                         int64_t total_tiles, cudaStream_t st) {
  if (total_tiles > 0x7fffffff) return cudaErrorInvalidConfiguration;
  k_gemm_simt_grouped<<<(unsigned)total_tiles, NT, 0, st>>>(d_probs, d_tile_start, nprob);
  return cudaGetLastError();
}
