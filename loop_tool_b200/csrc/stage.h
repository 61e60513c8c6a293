// Device-side stage descriptors shared by the host lowering (g++) and the
// kernels (nvcc).  Plain C structs: they are uploaded once per compiled
// loop tree and read by every launch.
#pragma once
#include <stdint.h>

#define LTB_MAXD 8    // iteration dims per stage (reference MAX_DEPTH is 8)
#define LTB_MAXL 8    // leaf loads per stage
#define LTB_MAXG 8    // bound guards per stage
#define LTB_MAXI 48   // VM instructions per stage
#define LTB_MAXC 8    // float constants per stage
#define LTB_MAXQ 64   // index-program words per stage (quasi-affine loads)
#define LTB_STACK 6   // VM stack depth
#define LTB_MAXBUF 48 // buffer slots per compiled nest (I/O + scratch)

// VM opcodes.  Binary ops pop b then a and push op(a, b), so programs are
// postfix in source order: "a b sub" computes a - b.
enum LtbVOp {
  LTB_V_LOAD = 0,  // push load[arg]
  LTB_V_CONST,     // push consts[arg]
  LTB_V_ADD,
  LTB_V_SUB,
  LTB_V_MUL,
  LTB_V_DIV,
  LTB_V_MIN,       // a < b ? a : b   (cpp.cpp:381-394 ternaries)
  LTB_V_MAX,       // a > b ? a : b
  LTB_V_EXP,
  LTB_V_LOG,
  LTB_V_SQRT,
  LTB_V_ABS,
  LTB_V_NEG,
  LTB_V_RECIP,     // 1 / a
  LTB_V_FOLD,      // acc = red_op(acc, pop())   (reduction stages)
};

enum LtbRedOp {
  LTB_R_NONE = 0,
  LTB_R_ADD,
  LTB_R_MUL,
  LTB_R_MAX,
  LTB_R_MIN,
  LTB_R_SUB,
  LTB_R_DIV,
};

// Index-program words for quasi-affine (div/mod) loads: postfix int64 ops.
enum LtbQOp {
  LTB_Q_COORD = 0,  // push x[arg]
  LTB_Q_CONST,      // push imm
  LTB_Q_ADD,
  LTB_Q_MUL,
  LTB_Q_DIV,        // C truncating division
  LTB_Q_MOD,
  LTB_Q_NEG,
  LTB_Q_MAX,
  LTB_Q_DIM,        // end of one buffer dim: check 0 <= v < imm (if arg),
                    // then flat = flat * imm + v
};

typedef struct {
  int32_t op;
  int32_t arg;
  int64_t imm;
} LtbQWord;

typedef struct {
  uint8_t op;
  uint8_t arg;
} LtbVInstr;

typedef struct {
  int64_t coef[LTB_MAXD];
  int64_t off;
  int64_t ub;  // valid iff 0 <= coef.x + off < ub
} LtbGuard;

enum LtbLoadMode {
  LTB_L_GENERAL = 0,  // coef . x + off (with guards / index program)
  LTB_L_LINEAR = 1,   // same flat index as the output: off + out_flat
  LTB_L_SCALAR = 2,   // one element broadcast: off
};

typedef struct {
  int32_t buf;      // buffer slot
  int32_t g0, ng;   // guards [g0, g0+ng) (affine loads)
  int32_t q0, nq;   // index program words (quasi-affine loads), nq == 0 => affine
  int32_t mode;     // LtbLoadMode
  int64_t coef[LTB_MAXD];  // flat index = coef.x + off (affine loads)
  int64_t off;
} LtbLoad;

typedef struct {
  int32_t ndim;   // total iteration dims
  int32_t nout;   // dims [0, nout) index the output, [nout, ndim) are reduced
  int32_t nload, ninstr, nguard, nconst, nq;
  int32_t red_op;     // LtbRedOp
  int32_t kahan;      // compensated summation for long add-reductions
  int32_t out_buf;
  int32_t split;      // >1: partial reductions go to partial_buf
  int32_t partial_buf;
  int32_t linear;     // elementwise stage whose loads are all LINEAR/SCALAR
  int32_t pattern;    // LtbPattern of a recognised fused chain (row_chain)
  int64_t size[LTB_MAXD];
  int64_t out_coef[LTB_MAXD];
  int64_t out_off;
  int64_t red_total;  // product of reduced sizes
  float red_init;
  float pad2_;
  LtbLoad loads[LTB_MAXL];
  LtbGuard guards[LTB_MAXG];
  LtbVInstr code[LTB_MAXI];
  float consts[LTB_MAXC];
  LtbQWord q[LTB_MAXQ];
  // 32-bit division by size[k] as (umulhi(n, mul) + n) >> shr
  // (Granlund-Montgomery), valid for n < 2^31
  uint32_t dm_mul[LTB_MAXD];
  uint32_t dm_shr[LTB_MAXD];
  int32_t small;      // every size and flat extent < 2^31: 32-bit indexing
  int32_t pad3_[3];   // keeps sizeof a multiple of 16 (int4 staging copies)
} LtbStage;

enum LtbPattern {
  LTB_P_NONE = 0,
  LTB_P_SOFTMAX = 1,  // m = max_n x; s = sum_n exp(x - m); y = exp(x - m) / s
};

// Buffer pointers of one run, passed by value to every launch.
typedef struct {
  float* p[LTB_MAXBUF];
} LtbBufTable;
