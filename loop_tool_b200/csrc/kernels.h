// Host-side launchers of the sm_100a kernel families.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "stage.h"

// Opts kernel fn into `bytes` of dynamic shared memory on the current
// device (the attribute is per device), once per kernel, device and larger
// size; thread-safe.
cudaError_t ltb_smem_optin(const void* fn, size_t bytes);

// Records `msg` as the calling thread's ltb_last_error() and returns code.
int ltb_set_last_error(int code, const char* msg);

// Launch schedule of one stage, chosen by the autotuner (zero fields keep
// the built-in heuristic).  cta_per_sm: grid = SMs x cta_per_sm CTAs
// (grid-stride kernels); threads: CTA size; variant: family-specific
// (row softmax: elements/threads pair; contraction: tile width 128/256).
struct LtbCfg {
  int cta_per_sm;
  int threads;
  int variant;
  // CTAs of the launch, fixed (a "parallel" loop annotation pins the
  // stage's thread count); 0: from cta_per_sm and the work
  int grid;
};


// (a) elementwise nests and (b) serial reductions
cudaError_t ltb_launch_nest(const LtbStage* d_stage, const LtbStage& h,
                            const LtbBufTable& bt, int sms, cudaStream_t st,
                            const LtbCfg& cfg);
// A plain linear elementwise map (each load reads the output's own flat
// index) run on the flat output range [lo, lo + n), lo a multiple of 8:
// lets host-staged runs pipeline copies and compute chunk by chunk.
int ltb_linear_range_ok(const LtbStage& h);
cudaError_t ltb_launch_linear_range(const LtbStage& h, const LtbBufTable& bt, int64_t lo,
                                    int64_t n, int sms, cudaStream_t st, const LtbCfg& cfg);
// (b) block-parallel reductions; splits > 1 writes split-K partials to the
// stage's partial buffer and combines them in order
cudaError_t ltb_launch_reduce(const LtbStage* d_stage, const LtbStage& h,
                              const LtbBufTable& bt, int splits, int sms,
                              cudaStream_t st, const LtbCfg& cfg);
// (b) fused per-row chain of stages (d_stages contiguous, final one
// elementwise; h_stages the host copies of the same stages)
cudaError_t ltb_launch_row_chain(const LtbStage* d_stages, const LtbStage* const* h_stages,
                                 int nsteps, const LtbBufTable& bt, int sms,
                                 cudaStream_t st, const LtbCfg& cfg, int* err);
// Candidate schedules the autotuner tries for a stage of a family (fills up
// to cap entries, returns the count).  The row-softmax variants depend on
// the row length.
int ltb_row_chain_candidates(const LtbStage* const* h_stages, int nsteps, LtbCfg* out, int cap);
int ltb_nest_candidates(const LtbStage& h, LtbCfg* out, int cap);
int ltb_reduce_candidates(const LtbStage& h, LtbCfg* out, int cap);

// (c) contractions.  Operand element (i, k) of A lives at
// a_rowoff[i] + a_koff[k] (B: b_rowoff[j] + b_koff[k]); guards are kept as
// per-row / per-k partial sums so padded convolutions gather implicitly.
struct LtbGemmOperand {
  const float* base;
  const int64_t* rowoff;  // [rows]
  const int64_t* koff;    // [K]
  // dense operands (no guards, rowoff[i] = i*ld_row, koff[k] = k*ld_k):
  // addresses are computed instead of read from the tables
  int dense;
  int64_t ld_row, ld_k;
  int nguard;
  const int32_t* grow;    // [nguard][rows] guard partial from the row coords
  const int32_t* gk;      // [nguard][K]   guard partial from the k coords
  const int32_t* gub;     // [nguard]      valid iff 0 <= grow + gk < gub
  int k32;                // every k offset (koff[k], or k * ld_k) fits in int32
};

struct LtbGemmProblem {
  LtbGemmOperand a, b;
  float* c;
  const int64_t* crow;  // [M] output offset per row
  const int64_t* ccol;  // [N] output offset per column
  int64_t M, N, K;
};

// FP32 CUDA-core path (every multiply and add rounded on its own, in k
// order: the reference C path's arithmetic): the "plain FP32" family.
// Operand tile loader forms (gemm_simt.cu); ltb_simt_mode picks the fastest
// one the operand's layout allows.
enum { kSimtGather = 0, kSimtVecK = 1, kSimtVecR = 2, kSimtGatherT = 3 };
constexpr int64_t kSimtMaxK = (int64_t(1) << 31) - 64;  // k indices are 32-bit
// a_side: the A operand (the gather form may use a shared per-k table).
int ltb_simt_mode(const LtbGemmOperand& op, int64_t rows, int64_t K, bool a_side);
// tile: 128 (128 x 128 CTA tiles, the loader forms above), 64 (64 x 64
// tiles for problems that 128-wide tiles leave SMs idle in), 0 = 64 when
// there are at most SMs / 4 tiles of 128 x 128, else 128.  Same bits either
// way.
cudaError_t ltb_launch_gemm_simt(const LtbGemmProblem& p, int sms,
                                 cudaStream_t st, int tile = 0);
int ltb_simt_tile(const LtbGemmProblem& p, int sms, int tile);
// Many problems in one launch: tile_start[i] = first 128 x 128 tile of
// problem i (device arrays), total_tiles tiles in all; modes = A form |
// B form << 4, a form every problem's operands allow (kSimtGather always
// does).
cudaError_t ltb_launch_gemm_simt_grouped(const LtbGemmProblem* d_probs,
                                         const int64_t* d_tile_start, int nprob,
                                         int64_t total_tiles, int modes, cudaStream_t st);

// Bounded-wait self-check (waitcheck.cu): one CTA whose mbarrier wait on a
// barrier nothing arrives at gives up after `limit` cycles, raising *err;
// status_host[2] = {wait completed, in-flight copy drained}.
cudaError_t ltb_launch_wait_check(int* err, long long limit, int* status_host, cudaStream_t st);
