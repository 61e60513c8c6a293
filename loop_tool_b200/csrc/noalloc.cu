// Row sums that allocate nothing: out[r] = sum_c x[r * cols + c].
//
// This is the split-K reduction of the reduction family (k_reduce_par with
// splits > 1 + k_reduce_combine, which keep their partials in the compiled
// object's scratch block) with its partial sums moved into one file-scope
// device array.  Some callers cannot allocate device memory when they call
// in: a serving loop that committed its whole HBM budget up front (an
// allocation there can fail under memory pressure, or synchronise the
// device in the middle of a latency-critical path), or a host framework
// that owns every device allocation itself.  They pass inputs and outputs
// only.
//
// Limits and sharing:
//  * the array holds LTB_NOALLOC_SCRATCH_FLOATS floats (4 MiB) and lives on
//    every GPU that loads this library until the process exits;
//  * rows * splits must fit in it; the entry point lowers `splits` to fit
//    and rejects rows > LTB_NOALLOC_SCRATCH_FLOATS;
//  * every call writes each partial it reads before reading it, so nothing
//    has to be cleared between calls, but all calls share the one array:
//    calls that overlap on the GPU (different streams, no ordering) race;
//  * the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress) -- make that first call before any stream
//    capture on that device.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/loop_tool_b200.h"
#include "compensated.cuh"
#include "kernels.h"

#define LTB_NOALLOC_SCRATCH_FLOATS (1 << 20)

static __device__ __align__(256) float g_noalloc_partials[LTB_NOALLOC_SCRATCH_FLOATS];

namespace {

struct KahanPart {
  float v, c;  // true sum ~= v - c
};

__device__ __forceinline__ KahanPart kp_combine(KahanPart a, KahanPart b) {
  ltbdev::comp_combine(a.v, a.c, b.v, b.c);
  return a;
}

// block (row, split): compensated sum of one contiguous chunk of one row
__global__ void __launch_bounds__(256)
    k_rowsum_partials(const float* __restrict__ x, int64_t rows, int64_t cols, int splits,
                      float* __restrict__ part) {
  __shared__ KahanPart sm[8];
  const int64_t chunk = (cols + splits - 1) / splits;
  for (int64_t row = blockIdx.x; row < rows; row += gridDim.x) {
    const int64_t c0 = (int64_t)blockIdx.y * chunk;
    const int64_t c1 = cols < c0 + chunk ? cols : c0 + chunk;
    const float* __restrict__ p = x + row * cols;
    KahanPart acc{0.f, 0.f};
    for (int64_t c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
      ltbdev::comp_add(acc.v, acc.c, __ldg(p + c));
    }
    for (int off = 16; off > 0; off >>= 1) {
      KahanPart o{__shfl_down_sync(0xffffffffu, acc.v, off),
                  __shfl_down_sync(0xffffffffu, acc.c, off)};
      if ((threadIdx.x & 31) + off < 32) acc = kp_combine(acc, o);
    }
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      KahanPart r = sm[0];
      for (int w = 1; w < (int)(blockDim.x >> 5); ++w) r = kp_combine(r, sm[w]);
      part[row * splits + blockIdx.y] = ltbdev::comp_value(r.v, r.c);
    }
    __syncthreads();
  }
}

// one thread per row: ordered compensated sum of its partials
__global__ void k_rowsum_combine(const float* __restrict__ part, int64_t rows, int splits,
                                 float* __restrict__ out) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < rows;
       r += (int64_t)gridDim.x * blockDim.x) {
    float acc = 0.f, c = 0.f;
    for (int s = 0; s < splits; ++s) ltbdev::comp_add(acc, c, part[r * splits + s]);
    out[r] = ltbdev::comp_value(acc, c);
  }
}

std::mutex g_mu;
void* g_addr[64] = {nullptr};  // device address of the array, per device

int noalloc_fail(int code, const std::string& msg) {
  return ltb_set_last_error(code, msg.c_str());
}

// Memory the kernels on device `dev` can read: managed memory, or device
// memory of `dev` itself (another GPU's memory would be a peer access).
bool on_device(const void* p, int dev) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeManaged || (a.type == cudaMemoryTypeDevice && a.device == dev);
}

}  // namespace

extern "C" int ltb_row_sum_noalloc(const float* x, int64_t rows, int64_t cols, float* out,
                                   void* stream) {
  if (!x || !out || rows < 0 || cols < 0)
    return noalloc_fail(LTB_ERR_INVALID, "null buffer or negative size");
  if (rows == 0) return LTB_OK;
  if (rows > LTB_NOALLOC_SCRATCH_FLOATS)
    return noalloc_fail(LTB_ERR_INVALID,
                        "rows (" + std::to_string(rows) + ") exceed the no-alloc scratch (" +
                            std::to_string(LTB_NOALLOC_SCRATCH_FLOATS) + " partial sums)");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
    return noalloc_fail(LTB_ERR_CUDA, "no current CUDA device");
  if (!on_device(x, dev) || !on_device(out, dev))
    return noalloc_fail(LTB_ERR_INVALID,
                        "managed buffers or device buffers of the current device required: "
                        "this entry point stages nothing");
  void* part = nullptr;
  {
    std::lock_guard<std::mutex> g(g_mu);
    if (!g_addr[dev]) {
      // host code only holds a stand-in for the array: ask for its address
      cudaError_t e = cudaGetSymbolAddress(&g_addr[dev], g_noalloc_partials);
      if (e != cudaSuccess) {
        g_addr[dev] = nullptr;
        return noalloc_fail(LTB_ERR_CUDA,
                            std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      }
    }
    part = g_addr[dev];
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // split-K width: ~4 CTAs per SM overall, >= 4096 columns per split, and
  // rows * splits within the array
  int64_t splits = (4LL * sms + rows - 1) / rows;
  if (splits > cols / 4096) splits = cols / 4096;
  if (splits > 2048) splits = 2048;
  if (splits > LTB_NOALLOC_SCRATCH_FLOATS / rows) splits = LTB_NOALLOC_SCRATCH_FLOATS / rows;
  if (splits < 1) splits = 1;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const unsigned gx = (unsigned)(rows < 65535 ? rows : 65535);
  k_rowsum_partials<<<dim3(gx, (unsigned)splits), 256, 0, st>>>(x, rows, cols, (int)splits,
                                                               static_cast<float*>(part));
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) {
    const unsigned g2 = (unsigned)((rows + 255) / 256 < 1024 ? (rows + 255) / 256 : 1024);
    k_rowsum_combine<<<g2, 256, 0, st>>>(static_cast<const float*>(part), rows, (int)splits,
                                         out);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) return noalloc_fail(LTB_ERR_CUDA, cudaGetErrorString(e));
  return LTB_OK;
}
