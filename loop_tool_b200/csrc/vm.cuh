// Device helpers shared by the elementwise / reduction kernel families:
// the stage-descriptor interpreter (a postfix stack machine held in fixed
// registers) and the fold operators.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "stage.h"

namespace ltbdev {

// Element ops with the reference semantics (cpp.cpp:172-270 emits them as C):
// min/max are the ternaries a<b?a:b / a>b?a:b.  Division, reciprocal and
// sqrt are IEEE correctly rounded (no fast-math), so they match the C path
// bit for bit; exp/log use the single-precision CUDA functions (a few ulp
// from the C path's double libm call rounded to float) -- the hot path has
// no FP64.
__device__ __forceinline__ float vm_bin(int op, float a, float b) {
  switch (op) {
    case LTB_V_ADD: return a + b;
    case LTB_V_SUB: return a - b;
    case LTB_V_MUL: return a * b;
    case LTB_V_DIV: return a / b;
    case LTB_V_MIN: return a < b ? a : b;
    default: return a > b ? a : b;  // LTB_V_MAX
  }
}

__device__ __forceinline__ float vm_un(int op, float a) {
  switch (op) {
    case LTB_V_EXP: return expf(a);
    case LTB_V_LOG: return logf(a);
    case LTB_V_SQRT: return sqrtf(a);
    case LTB_V_ABS: return fabsf(a);
    case LTB_V_NEG: return -a;
    default: return 1.0f / a;  // LTB_V_RECIP
  }
}

__device__ __forceinline__ float fold(int red_op, float acc, float x) {
  switch (red_op) {
    case LTB_R_ADD: return acc + x;
    case LTB_R_MUL: return acc * x;
    case LTB_R_MAX: return acc > x ? acc : x;
    case LTB_R_MIN: return acc < x ? acc : x;
    case LTB_R_SUB: return acc - x;
    default: return acc / x;  // LTB_R_DIV
  }
}

// Quasi-affine index program: returns false when a guarded dim is out of
// bounds (the reference reads 0 there, cpp.cpp:103-106).
__device__ __forceinline__ bool qindex(const LtbStage& S, const LtbLoad& L,
                                       const int64_t* x, int64_t* flat_out) {
  int64_t st[8];
  int sp = 0;
  int64_t flat = 0;
  for (int i = L.q0; i < L.q0 + L.nq; ++i) {
    const LtbQWord w = S.q[i];
    switch (w.op) {
      case LTB_Q_COORD: st[sp++] = x[w.arg]; break;
      case LTB_Q_CONST: st[sp++] = w.imm; break;
      case LTB_Q_NEG: st[sp - 1] = -st[sp - 1]; break;
      case LTB_Q_DIM: {
        int64_t v = st[--sp];
        if (w.arg && (v < 0 || v >= w.imm)) return false;
        flat = flat * w.imm + v;
        break;
      }
      default: {
        int64_t b = st[--sp];
        int64_t a = st[sp - 1];
        int64_t r;
        switch (w.op) {
          case LTB_Q_ADD: r = a + b; break;
          case LTB_Q_MUL: r = a * b; break;
          case LTB_Q_DIV: r = b ? a / b : 0; break;
          case LTB_Q_MOD: r = b ? a % b : 0; break;
          default: r = a > b ? a : b; break;
        }
        st[sp - 1] = r;
      }
    }
  }
  *flat_out = flat;
  return true;
}

// Scalar load of load `li` at full coordinates x.
__device__ __forceinline__ float load_at(const LtbStage& S, const LtbBufTable& bt,
                                         int li, const int64_t* x) {
  const LtbLoad& L = S.loads[li];
  if (L.nq) {
    int64_t flat;
    if (!qindex(S, L, x, &flat)) return 0.f;
    return __ldg(bt.p[L.buf] + flat);
  }
  int64_t idx = L.off;
  for (int k = 0; k < S.ndim; ++k) idx += L.coef[k] * x[k];
  for (int gi = L.g0; gi < L.g0 + L.ng; ++gi) {
    const LtbGuard& G = S.guards[gi];
    int64_t gv = G.off;
    for (int k = 0; k < S.ndim; ++k) gv += G.coef[k] * x[k];
    if (gv < 0 || gv >= G.ub) return 0.f;
  }
  return bt.p[L.buf][idx];
}

// Evaluate the stage program at one point.  Returns the value left on the
// stack (elementwise stages) and folds FOLD operands into *acc.
__device__ __forceinline__ float vm_eval_point(const LtbStage& S,
                                               const LtbBufTable& bt,
                                               const int64_t* x, float* acc) {
  float s0 = 0, s1 = 0, s2 = 0, s3 = 0, s4 = 0, s5 = 0;
  for (int i = 0; i < S.ninstr; ++i) {
    const LtbVInstr in = S.code[i];
    const int op = in.op;
    if (op == LTB_V_LOAD || op == LTB_V_CONST) {
      float v = op == LTB_V_LOAD ? load_at(S, bt, in.arg, x) : S.consts[in.arg];
      s5 = s4; s4 = s3; s3 = s2; s2 = s1; s1 = s0; s0 = v;
    } else if (op == LTB_V_FOLD) {
      *acc = fold(S.red_op, *acc, s0);
      s0 = s1; s1 = s2; s2 = s3; s3 = s4; s4 = s5;
    } else if (op >= LTB_V_EXP) {
      s0 = vm_un(op, s0);
    } else {
      s0 = vm_bin(op, s1, s0);
      s1 = s2; s2 = s3; s3 = s4; s4 = s5;
    }
  }
  return s0;
}

}  // namespace ltbdev
