// Synthetic request inputs for the native serving loop (serve.cpp): a
// buffer of rows x cols FP32 values, row-major, whose top-left true_rows x
// true_cols block holds seeded normal values times `scale` and whose other
// elements (shape-bucket padding) are zero.  Element (i, j) of the block
// takes the value of counter i * true_cols + j, so a request's inputs are
// the same whether or not its buffer is padded.
//
// Counter-based normals: SplitMix64 (Steele, Lea, Flood, "Fast splittable
// pseudorandom number generators", 2014) hashes (seed, counter) into two
// 24-bit uniforms, the Box-Muller transform turns them into one N(0, 1)
// value.
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.h"

namespace {

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

__device__ __forceinline__ float seeded_normal(uint64_t seed, uint64_t i) {
  const uint64_t h = splitmix64(seed ^ splitmix64(i));
  // u1 in (0, 1], u2 in [0, 1): 24-bit uniforms
  const float u1 = ((float)(h >> 40) + 1.0f) * (1.0f / 16777216.0f);
  const float u2 = (float)((h >> 16) & 0xFFFFFF) * (1.0f / 16777216.0f);
  return sqrtf(-2.0f * logf(u1)) * cospif(2.0f * u2);
}

__global__ void k_fill_block(float* __restrict__ x, int64_t rows, int64_t cols, int64_t trows,
                             int64_t tcols, uint64_t seed, float scale) {
  const int64_t n = rows * cols;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e / cols, j = e - i * cols;
    x[e] = (i < trows && j < tcols) ? scale * seeded_normal(seed, (uint64_t)(i * tcols + j))
                                    : 0.f;
  }
}

}  // namespace

cudaError_t ltb_launch_fill_block(float* x, int64_t rows, int64_t cols, int64_t true_rows,
                                  int64_t true_cols, uint64_t seed, float scale, int sms,
                                  cudaStream_t st) {
  const int64_t n = rows * cols;
  if (n <= 0) return cudaSuccess;
  int64_t blocks = (n + 255) / 256;
  if (blocks > (int64_t)sms * 16) blocks = (int64_t)sms * 16;
  k_fill_block<<<(unsigned)blocks, 256, 0, st>>>(x, rows, cols, true_rows, true_cols, seed,
                                                  scale);
  return cudaGetLastError();
}
