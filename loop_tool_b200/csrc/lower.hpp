// Lowering: serialized IR -> a plan of kernel launches.
//
// The plan computes the dataflow semantics of the IR, which every legal
// LoopTree over it computes too: element values follow the reference "cpp"
// backend (cpp.cpp:172-270: left folds, ternary min/max, out-of-bounds reads
// as 0), index equations follow Compiler::gen_index_equations
// (compile.cpp:611-756).  The LoopTree schedule does not change values
// beyond what the reference's own order does (reductions fold in the
// node's loop order); its loop annotations pin launch choices (StagePins).
#pragma once

#include <string>
#include <vector>

#include "ir.hpp"
#include "stage.h"

namespace ltb {

enum class Family : int {
  elementwise = 0,   // (a) quasi-affine elementwise / broadcast / view nest
  reduce_serial,     // (b) one thread per output, serial over the window
  reduce_parallel,   // (b) one block per output, warp-shuffle + smem tree
  reduce_split,      // (b) split-K partials + ordered combine
  row_chain,         // (b) fused per-row reduction chain (softmax-like)
  contraction,       // (c) matmul / implicit-GEMM conv on tensor cores
};
const char* family_name(Family f);

enum class Precision : int { fp32 = 0, bf16 = 1, bf16x3 = 2, bf16x4 = 3, bf16x6 = 4 };

struct BufferInfo {
  int slot = -1;
  std::vector<int> layout;  // IR vars, outermost first (row-major)
  std::vector<int64_t> sizes;
  int64_t elems = 1;
  bool scratch = false;
};

// A dense contraction C[b, m, n] = sum_k A[b, m, k] * B[b, k, n] in which
// every operand element address is affine in (b, m, k) / (b, k, n)
// (possibly guarded, e.g. padded convolution).
struct Contraction {
  std::vector<int> bvars, mvars, nvars, kvars;  // IR vars per role
  int64_t B = 1, M = 1, N = 1, K = 1;
  // load descriptors in the stage dim order [bvars, mvars, nvars, kvars]
  int a_load = -1, b_load = -1;
  bool a_guarded = false, b_guarded = false;
};

// What the loop annotations of a stage's node ask for (LoopTree loop
// annotations: IR::annotate_loop, ir.h:183-195, set by annotate(),
// mutate.cpp:694-712; the reference's vocabulary is "parallel", "unroll",
// "vectorize" and "[backend]").  A loop's iteration count is its size plus
// one when it has a tail.
struct StagePins {
  // "parallel" loops over the stage's output vars: the product of their
  // iteration counts is the number of device threads the stage runs with
  // (CTAs x CTA size); the innermost such loop, when there are two or more,
  // is the CTA size.  0: free.
  int64_t parallel_out = 0;
  int cta_threads = 0;
  // "parallel" loops over reduced vars: the width of the parallel
  // reduction (threads per output, or split-K partials).  0: free.
  int64_t parallel_red = 0;
  // "unroll": iteration count of the innermost unrolled loop (items per
  // thread where the family has that choice).  0: free.
  int unroll = 0;
  bool any() const { return parallel_out || parallel_red || unroll; }
  std::string text;  // what the plan made of the annotations
};

struct PlanStage {
  Family family = Family::elementwise;
  StagePins pins;
  int node = -1;
  std::vector<int> dim_vars;  // stage iteration vars: outputs then reduced
  LtbStage dev{};             // device descriptor
  int rows_from = -1;         // row_chain: index of first fused stage
  Contraction con;            // contraction details (family == contraction)
  std::string text;           // human-readable summary
};

struct LowerOptions {
  Precision precision = Precision::fp32;
  bool fuse_rows = true;
  bool use_tensor_cores = true;
  int kahan_threshold = 65536;
};

struct Plan {
  int n_in = 0, n_out = 0;
  std::vector<int64_t> io_elems;       // per I/O slot (inputs then outputs)
  std::vector<int64_t> scratch_elems;  // per scratch slot
  std::vector<PlanStage> stages;
  std::vector<std::vector<int>> row_groups;  // stage indices fused per group
  int64_t algorithmic_bytes = 0;  // compulsory I/O bytes of one run
  double flops = 0;               // arithmetic (2*MNK for contractions)
  std::string dump;
  int num_slots() const { return n_in + n_out + (int)scratch_elems.size(); }
};

Plan lower(const IRGraph& g, const LowerOptions& opt);

}  // namespace ltb
