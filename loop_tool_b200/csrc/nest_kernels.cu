// Families (a) and (b): elementwise / broadcast / view nests and reductions,
// interpreted from LtbStage descriptors.  All of them are HBM-bound, so the
// design points are coalescing, 128-bit accesses along the innermost output
// dim, and grids sized in multiples of the 148 SMs.
#include <cfloat>

#include "kernels.h"
#include "vm.cuh"

using namespace ltbdev;

namespace {

__device__ __forceinline__ void load_stage(const LtbStage* __restrict__ g,
                                           LtbStage& s) {
  const int4* src = reinterpret_cast<const int4*>(g);
  int4* dst = reinterpret_cast<int4*>(&s);
  for (int i = threadIdx.x; i < (int)(sizeof(LtbStage) / 16); i += blockDim.x)
    dst[i] = src[i];
  __syncthreads();
}

template <int VEC>
struct Lanes {
  float v[VEC];
};

// Load `li` for VEC consecutive values of the innermost output dim ki.
template <int VEC>
__device__ __forceinline__ Lanes<VEC> load_lanes(const LtbStage& S,
                                                 const LtbBufTable& bt, int li,
                                                 int64_t* x, int ki, int nv) {
  Lanes<VEC> r;
  const LtbLoad& L = S.loads[li];
  const float* __restrict__ p = bt.p[L.buf];
  if (L.nq) {
    const int64_t x0 = ki >= 0 ? x[ki] : 0;
#pragma unroll
    for (int j = 0; j < VEC; ++j) {
      r.v[j] = 0.f;
      if (j < nv) {
        if (ki >= 0) x[ki] = x0 + j;
        int64_t flat;
        if (qindex(S, L, x, &flat)) r.v[j] = p[flat];
      }
    }
    if (ki >= 0) x[ki] = x0;
    return r;
  }
  int64_t base = L.off;
  for (int k = 0; k < S.ndim; ++k) base += L.coef[k] * x[k];
  const int64_t step = ki >= 0 ? L.coef[ki] : 0;
  if (L.ng == 0) {
    if (VEC == 4 && step == 1 && nv == 4 && (base & 3) == 0) {
      float4 q = *reinterpret_cast<const float4*>(p + base);
      r.v[0] = q.x;
      r.v[1 % VEC] = q.y;
      r.v[2 % VEC] = q.z;
      r.v[3 % VEC] = q.w;
      return r;
    }
    if (step == 0) {
      float s = p[base];
#pragma unroll
      for (int j = 0; j < VEC; ++j) r.v[j] = s;
      return r;
    }
#pragma unroll
    for (int j = 0; j < VEC; ++j) r.v[j] = j < nv ? p[base + j * step] : 0.f;
    return r;
  }
  bool ok[VEC];
#pragma unroll
  for (int j = 0; j < VEC; ++j) ok[j] = j < nv;
  for (int gi = L.g0; gi < L.g0 + L.ng; ++gi) {
    const LtbGuard& G = S.guards[gi];
    int64_t gv = G.off;
    for (int k = 0; k < S.ndim; ++k) gv += G.coef[k] * x[k];
    const int64_t gs = ki >= 0 ? G.coef[ki] : 0;
#pragma unroll
    for (int j = 0; j < VEC; ++j) {
      int64_t v = gv + j * gs;
      ok[j] = ok[j] && v >= 0 && v < G.ub;
    }
  }
#pragma unroll
  for (int j = 0; j < VEC; ++j) r.v[j] = ok[j] ? p[base + j * step] : 0.f;
  return r;
}

// Generic nest kernel: elementwise stages and serial reductions.  One thread
// produces VEC consecutive outputs along the innermost output dim and
// walks the reduced dims in order (exact sequential fold semantics).
template <int VEC>
__global__ void __launch_bounds__(256)
    k_nest(const LtbStage* __restrict__ gst, LtbBufTable bt) {
  __shared__ __align__(16) LtbStage S;
  load_stage(gst, S);
  const int nd = S.ndim, no = S.nout;
  const int ki = no - 1;
  const int64_t inner = no ? S.size[ki] : 1;
  const int64_t nvec = (inner + VEC - 1) / VEC;
  int64_t outer = 1;
  for (int k = 0; k < ki; ++k) outer *= S.size[k];
  const int64_t total = outer * nvec;
  const bool has_red = nd > no;
  float* __restrict__ out = bt.p[S.out_buf];
  const int64_t ostep = ki >= 0 ? S.out_coef[ki] : 0;

  for (int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; w < total;
       w += (int64_t)gridDim.x * blockDim.x) {
    int64_t x[LTB_MAXD];
    int64_t o = w / nvec;
    const int64_t iv = w - o * nvec;
    for (int k = ki - 1; k >= 0; --k) {
      const int64_t q = o / S.size[k];
      x[k] = o - q * S.size[k];
      o = q;
    }
    if (ki >= 0) x[ki] = iv * VEC;
    const int nv = (int)(inner - iv * VEC < VEC ? inner - iv * VEC : VEC);
    for (int k = no; k < nd; ++k) x[k] = 0;

    float acc[VEC], comp[VEC];
#pragma unroll
    for (int j = 0; j < VEC; ++j) {
      acc[j] = S.red_init;
      comp[j] = 0.f;
    }
    Lanes<VEC> s0{}, s1{}, s2{}, s3{}, s4{}, s5{};
    const int64_t R = has_red ? S.red_total : 1;
    for (int64_t r = 0; r < R; ++r) {
      for (int i = 0; i < S.ninstr; ++i) {
        const LtbVInstr in = S.code[i];
        const int op = in.op;
        if (op == LTB_V_LOAD || op == LTB_V_CONST) {
          Lanes<VEC> t;
          if (op == LTB_V_LOAD) {
            t = load_lanes<VEC>(S, bt, in.arg, x, ki, nv);
          } else {
#pragma unroll
            for (int j = 0; j < VEC; ++j) t.v[j] = S.consts[in.arg];
          }
          s5 = s4; s4 = s3; s3 = s2; s2 = s1; s1 = s0; s0 = t;
        } else if (op == LTB_V_FOLD) {
          if (S.kahan) {
#pragma unroll
            for (int j = 0; j < VEC; ++j) {  // Kahan-Babuska summation
              const float y = s0.v[j] - comp[j];
              const float t = acc[j] + y;
              comp[j] = (t - acc[j]) - y;
              acc[j] = t;
            }
          } else {
#pragma unroll
            for (int j = 0; j < VEC; ++j) acc[j] = fold(S.red_op, acc[j], s0.v[j]);
          }
          s0 = s1; s1 = s2; s2 = s3; s3 = s4; s4 = s5;
        } else if (op >= LTB_V_EXP) {
#pragma unroll
          for (int j = 0; j < VEC; ++j) s0.v[j] = vm_un(op, s0.v[j]);
        } else {
#pragma unroll
          for (int j = 0; j < VEC; ++j) s0.v[j] = vm_bin(op, s1.v[j], s0.v[j]);
          s1 = s2; s2 = s3; s3 = s4; s4 = s5;
        }
      }
      // odometer over the reduced dims, innermost fastest
      for (int k = nd - 1; k >= no; --k) {
        if (++x[k] < S.size[k]) break;
        x[k] = 0;
      }
    }
    int64_t obase = S.out_off;
    for (int k = 0; k < no; ++k) obase += S.out_coef[k] * x[k];
    float res[VEC];
#pragma unroll
    for (int j = 0; j < VEC; ++j) res[j] = has_red ? acc[j] : s0.v[j];
    if (VEC == 4 && ostep == 1 && nv == 4 && (obase & 3) == 0) {
      *reinterpret_cast<float4*>(out + obase) =
          make_float4(res[0], res[1 % VEC], res[2 % VEC], res[3 % VEC]);
    } else {
#pragma unroll
      for (int j = 0; j < VEC; ++j)
        if (j < nv) out[obase + j * ostep] = res[j];
    }
  }
}

// ---------------------------------------------------------------- ordered
// Partial state of a parallel fold.  max/min keep the index of the value so
// that combining partials reproduces the sequential ternary fold exactly:
// `acc = acc > x ? acc : x` keeps the LAST of equal values (which decides
// +0 vs -0).  NaN inputs break that order-independence, so a NaN sends the
// output back to a sequential pass.
struct Part {
  float v;
  float c;      // Kahan compensation (add)
  int64_t i;    // index of v (max/min)
  int nan;
};

__device__ __forceinline__ Part part_init(int op, float init) {
  Part p;
  p.v = init;
  p.c = 0.f;
  p.i = -1;
  p.nan = 0;
  return p;
}

__device__ __forceinline__ void part_add(Part& p, int op, int kahan, float x,
                                         int64_t idx) {
  switch (op) {
    case LTB_R_ADD:
      if (kahan) {
        const float y = x - p.c;
        const float t = p.v + y;
        p.c = (t - p.v) - y;
        p.v = t;
      } else {
        p.v += x;
      }
      break;
    case LTB_R_MUL: p.v *= x; break;
    case LTB_R_MAX:
      if (isnan(x)) p.nan = 1;
      else if (!(p.v > x)) { p.v = x; p.i = idx; }
      break;
    default:  // LTB_R_MIN
      if (isnan(x)) p.nan = 1;
      else if (!(p.v < x)) { p.v = x; p.i = idx; }
      break;
  }
}

// combine a (covering earlier or interleaved indices) with b
__device__ __forceinline__ Part part_combine(int op, Part a, Part b) {
  Part r = a;
  r.nan = a.nan | b.nan;
  switch (op) {
    case LTB_R_ADD: {
      // TwoSum of the running values; their rounding error joins the
      // compensation terms (true sum ~= v - c)
      const float s = a.v + b.v;
      const float bp = s - a.v;
      const float e = (a.v - (s - bp)) + (b.v - bp);
      r.c = a.c + b.c - e;
      r.v = s;
      break;
    }
    case LTB_R_MUL: r.v = a.v * b.v; break;
    case LTB_R_MAX: {
      bool take_b = b.v > a.v || (b.v == a.v && b.i > a.i);
      if (take_b) { r.v = b.v; r.i = b.i; }
      break;
    }
    default: {
      bool take_b = b.v < a.v || (b.v == a.v && b.i > a.i);
      if (take_b) { r.v = b.v; r.i = b.i; }
      break;
    }
  }
  return r;
}

__device__ __forceinline__ Part shfl_part(Part p, int off) {
  Part q;
  q.v = __shfl_down_sync(0xffffffffu, p.v, off);
  q.c = __shfl_down_sync(0xffffffffu, p.c, off);
  q.i = __shfl_down_sync(0xffffffffu, p.i, off);
  q.nan = __shfl_down_sync(0xffffffffu, p.nan, off);
  return q;
}

// Block-wide ordered reduction; result valid in thread 0.
__device__ Part block_reduce(int op, Part p, Part* sm) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int off = 16; off > 0; off >>= 1) {
    Part q = shfl_part(p, off);
    if (lane + off < 32) p = part_combine(op, p, q);
  }
  if (lane == 0) sm[wid] = p;
  __syncthreads();
  if (wid == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    p = lane < nw ? sm[lane] : sm[0];
    for (int off = 16; off > 0; off >>= 1) {
      Part q = shfl_part(p, off);
      if (lane + off < nw) p = part_combine(op, p, q);
    }
  }
  __syncthreads();
  return p;
}

__device__ __forceinline__ void set_red_coords(const LtbStage& S, int64_t r,
                                               int64_t* x) {
  for (int k = S.ndim - 1; k >= S.nout; --k) {
    const int64_t q = r / S.size[k];
    x[k] = r - q * S.size[k];
    r = q;
  }
}

__device__ __forceinline__ void set_out_coords(const LtbStage& S, int64_t o,
                                               int64_t* x) {
  for (int k = S.nout - 1; k >= 0; --k) {
    const int64_t q = o / S.size[k];
    x[k] = o - q * S.size[k];
    o = q;
  }
}

// Sequential fold of one output (exact reference order), used when NaNs
// make the parallel order matter.
__device__ float serial_fold(const LtbStage& S, const LtbBufTable& bt,
                             int64_t* x, int64_t r0, int64_t r1, float acc) {
  for (int64_t r = r0; r < r1; ++r) {
    set_red_coords(S, r, x);
    vm_eval_point(S, bt, x, &acc);
  }
  return acc;
}

// One block per output point (grid-strided), threads split the reduced
// range; gridDim.y > 1 splits it further into partials (split-K).
__global__ void __launch_bounds__(256)
    k_reduce_par(const LtbStage* __restrict__ gst, LtbBufTable bt,
                 int64_t nout_total) {
  __shared__ __align__(16) LtbStage S;
  __shared__ Part sm[32];
  load_stage(gst, S);
  const int64_t R = S.red_total;
  const int splits = gridDim.y;
  const int64_t chunk = (R + splits - 1) / splits;
  const int64_t r0 = blockIdx.y * chunk;
  const int64_t r1 = R < r0 + chunk ? R : r0 + chunk;
  for (int64_t o = blockIdx.x; o < nout_total; o += gridDim.x) {
    int64_t x[LTB_MAXD];
    set_out_coords(S, o, x);
    Part p = part_init(S.red_op, S.red_init);
    if (S.red_op == LTB_R_ADD) p.v = 0.f;
    if (S.red_op == LTB_R_MUL) p.v = 1.f;
    for (int64_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
      set_red_coords(S, r, x);
      // every FOLD feeds one reduction input term into the partial
      float s0 = 0, s1 = 0, s2 = 0, s3 = 0, s4 = 0, s5 = 0;
      for (int i = 0; i < S.ninstr; ++i) {
        const LtbVInstr in = S.code[i];
        const int op = in.op;
        if (op == LTB_V_LOAD || op == LTB_V_CONST) {
          float v = op == LTB_V_LOAD ? load_at(S, bt, in.arg, x) : S.consts[in.arg];
          s5 = s4; s4 = s3; s3 = s2; s2 = s1; s1 = s0; s0 = v;
        } else if (op == LTB_V_FOLD) {
          part_add(p, S.red_op, S.kahan, s0, r);
          s0 = s1; s1 = s2; s2 = s3; s3 = s4; s4 = s5;
        } else if (op >= LTB_V_EXP) {
          s0 = vm_un(op, s0);
        } else {
          s0 = vm_bin(op, s1, s0);
          s1 = s2; s2 = s3; s3 = s4; s4 = s5;
        }
      }
    }
    p = block_reduce(S.red_op, p, sm);
    if (threadIdx.x == 0) {
      float res;
      const bool ordered = S.red_op == LTB_R_MAX || S.red_op == LTB_R_MIN;
      if (ordered && p.nan) {
        res = serial_fold(S, bt, x, r0, r1, splits > 1 ? p.v : S.red_init);
        if (splits > 1) res = NAN;  // split partials never carry max/min
      } else if (ordered) {
        res = fold(S.red_op, S.red_init, p.v);
        if (p.i < 0) res = S.red_init;
      } else if (splits == 1) {
        res = fold(S.red_op, S.red_init, p.v - p.c);
      } else {
        res = p.v - p.c;
      }
      if (splits == 1) {
        int64_t ob = S.out_off;
        for (int k = 0; k < S.nout; ++k) ob += S.out_coef[k] * x[k];
        bt.p[S.out_buf][ob] = res;
      } else {
        bt.p[S.partial_buf][o * splits + blockIdx.y] = res;
      }
    }
    __syncthreads();
  }
}

// Ordered combine of split-K partials (add / mul only).
__global__ void k_reduce_combine(const LtbStage* __restrict__ gst,
                                 LtbBufTable bt, int64_t nout_total,
                                 int splits) {
  __shared__ __align__(16) LtbStage S;
  load_stage(gst, S);
  for (int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
       o < nout_total; o += (int64_t)gridDim.x * blockDim.x) {
    const float* part = bt.p[S.partial_buf] + o * splits;
    float acc = S.red_init, c = 0.f;
    for (int s = 0; s < splits; ++s) {
      if (S.red_op == LTB_R_ADD) {
        const float y = part[s] - c;
        const float t = acc + y;
        c = (t - acc) - y;
        acc = t;
      } else {
        acc = fold(S.red_op, acc, part[s]);
      }
    }
    int64_t x[LTB_MAXD];
    set_out_coords(S, o, x);
    int64_t ob = S.out_off;
    for (int k = 0; k < S.nout; ++k) ob += S.out_coef[k] * x[k];
    bt.p[S.out_buf][ob] = acc;
  }
}

// ------------------------------------------------------------- row chain
// A chain of stages over the same rows: reductions over the inner dim that
// produce per-row scalars, ending in a per-element output (row softmax:
// max, sum(exp(x - max)), exp(x - max) / sum).  One CTA owns one row for
// the whole chain; per-row scalars stay in shared memory and the row's
// later reads hit L1/L2, so HBM sees one read and one write per element.
constexpr int kMaxChain = 6;

__device__ __forceinline__ float chain_load(const LtbStage& S,
                                            const LtbBufTable& bt, int li,
                                            const int64_t* x, const int* rs_slot,
                                            const float* rs_val, int nrs) {
  const int b = S.loads[li].buf;
  for (int i = 0; i < nrs; ++i)
    if (rs_slot[i] == b) return rs_val[i];
  return load_at(S, bt, li, x);
}

__global__ void __launch_bounds__(512)
    k_row_chain(const LtbStage* __restrict__ gst, int nsteps, LtbBufTable bt,
                int64_t nrows) {
  __shared__ __align__(16) LtbStage S[kMaxChain];
  __shared__ Part sm[32];
  __shared__ int rs_slot[kMaxChain];
  __shared__ float rs_val[kMaxChain];
  {
    const int4* src = reinterpret_cast<const int4*>(gst);
    int4* dst = reinterpret_cast<int4*>(S);
    const int n16 = nsteps * (int)(sizeof(LtbStage) / 16);
    for (int i = threadIdx.x; i < n16; i += blockDim.x) dst[i] = src[i];
    __syncthreads();
  }
  const LtbStage& F = S[nsteps - 1];  // final elementwise stage
  const int nrow_dims = F.nout - 1;
  const int64_t inner = F.size[F.nout - 1];
  for (int64_t row = blockIdx.x; row < nrows; row += gridDim.x) {
    int64_t x[LTB_MAXD];
    {
      int64_t o = row;
      for (int k = nrow_dims - 1; k >= 0; --k) {
        const int64_t q = o / F.size[k];
        x[k] = o - q * F.size[k];
        o = q;
      }
    }
    int nrs = 0;
    for (int s = 0; s < nsteps; ++s) {
      const LtbStage& T = S[s];
      if (s < nsteps - 1) {
        Part p = part_init(T.red_op, T.red_init);
        if (T.red_op == LTB_R_ADD) p.v = 0.f;
        if (T.red_op == LTB_R_MUL) p.v = 1.f;
        for (int64_t n = threadIdx.x; n < inner; n += blockDim.x) {
          x[nrow_dims] = n;
          float s0 = 0, s1 = 0, s2 = 0, s3 = 0, s4 = 0, s5 = 0;
          for (int i = 0; i < T.ninstr; ++i) {
            const LtbVInstr in = T.code[i];
            const int op = in.op;
            if (op == LTB_V_LOAD || op == LTB_V_CONST) {
              float v = op == LTB_V_LOAD
                            ? chain_load(T, bt, in.arg, x, rs_slot, rs_val, nrs)
                            : T.consts[in.arg];
              s5 = s4; s4 = s3; s3 = s2; s2 = s1; s1 = s0; s0 = v;
            } else if (op == LTB_V_FOLD) {
              part_add(p, T.red_op, T.kahan, s0, n);
              s0 = s1; s1 = s2; s2 = s3; s3 = s4; s4 = s5;
            } else if (op >= LTB_V_EXP) {
              s0 = vm_un(op, s0);
            } else {
              s0 = vm_bin(op, s1, s0);
              s1 = s2; s2 = s3; s3 = s4; s4 = s5;
            }
          }
        }
        p = block_reduce(T.red_op, p, sm);
        if (threadIdx.x == 0) {
          float res;
          const bool ordered = T.red_op == LTB_R_MAX || T.red_op == LTB_R_MIN;
          if (ordered && p.nan) {
            res = T.red_init;
            for (int64_t n = 0; n < inner; ++n) {
              x[nrow_dims] = n;
              float a = res;
              // sequential pass; scratch scalars from earlier steps
              float s0 = 0, s1 = 0, s2 = 0, s3 = 0, s4 = 0, s5 = 0;
              for (int i = 0; i < T.ninstr; ++i) {
                const LtbVInstr in = T.code[i];
                const int op = in.op;
                if (op == LTB_V_LOAD || op == LTB_V_CONST) {
                  float v = op == LTB_V_LOAD ? chain_load(T, bt, in.arg, x, rs_slot,
                                                          rs_val, nrs)
                                             : T.consts[in.arg];
                  s5 = s4; s4 = s3; s3 = s2; s2 = s1; s1 = s0; s0 = v;
                } else if (op == LTB_V_FOLD) {
                  a = fold(T.red_op, a, s0);
                  s0 = s1; s1 = s2; s2 = s3; s3 = s4; s4 = s5;
                } else if (op >= LTB_V_EXP) {
                  s0 = vm_un(op, s0);
                } else {
                  s0 = vm_bin(op, s1, s0);
                  s1 = s2; s2 = s3; s3 = s4; s4 = s5;
                }
              }
              res = a;
            }
          } else if (ordered) {
            res = p.i < 0 ? T.red_init : fold(T.red_op, T.red_init, p.v);
          } else {
            res = fold(T.red_op, T.red_init, p.v - p.c);
          }
          rs_slot[nrs] = T.out_buf;
          rs_val[nrs] = res;
          int64_t ob = T.out_off;
          for (int k = 0; k < T.nout; ++k) ob += T.out_coef[k] * x[k];
          bt.p[T.out_buf][ob] = res;  // visible to consumers outside the chain
        }
        __syncthreads();
        nrs++;
      } else {
        float* __restrict__ out = bt.p[T.out_buf];
        int64_t obase = T.out_off;
        for (int k = 0; k < nrow_dims; ++k) obase += T.out_coef[k] * x[k];
        const int64_t ostep = T.out_coef[nrow_dims];
        for (int64_t n = threadIdx.x; n < inner; n += blockDim.x) {
          x[nrow_dims] = n;
          float s0 = 0, s1 = 0, s2 = 0, s3 = 0, s4 = 0, s5 = 0;
          for (int i = 0; i < T.ninstr; ++i) {
            const LtbVInstr in = T.code[i];
            const int op = in.op;
            if (op == LTB_V_LOAD || op == LTB_V_CONST) {
              float v = op == LTB_V_LOAD
                            ? chain_load(T, bt, in.arg, x, rs_slot, rs_val, nrs)
                            : T.consts[in.arg];
              s5 = s4; s4 = s3; s3 = s2; s2 = s1; s1 = s0; s0 = v;
            } else if (op >= LTB_V_EXP) {
              s0 = vm_un(op, s0);
            } else {
              s0 = vm_bin(op, s1, s0);
              s1 = s2; s2 = s3; s3 = s4; s4 = s5;
            }
          }
          out[obase + n * ostep] = s0;
        }
        __syncthreads();
      }
    }
  }
}

}  // namespace

// ------------------------------------------------------------ launchers
static int grid_for(int64_t work, int threads, int sms) {
  int64_t blocks = (work + threads - 1) / threads;
  const int64_t cap = (int64_t)sms * 16;  // 16 resident 256-thread CTAs/SM
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  return (int)blocks;
}

cudaError_t ltb_launch_nest(const LtbStage* d_stage, const LtbStage& h,
                            const LtbBufTable& bt, int sms, cudaStream_t st) {
  const int no = h.nout;
  const int64_t inner = no ? h.size[no - 1] : 1;
  int64_t outer = 1;
  for (int k = 0; k < no - 1; ++k) outer *= h.size[k];
  const bool vec = inner >= 4;
  const int64_t work = outer * (vec ? (inner + 3) / 4 : inner);
  const int threads = 256;
  const int grid = grid_for(work, threads, sms);
  if (vec)
    k_nest<4><<<grid, threads, 0, st>>>(d_stage, bt);
  else
    k_nest<1><<<grid, threads, 0, st>>>(d_stage, bt);
  return cudaGetLastError();
}

cudaError_t ltb_launch_reduce(const LtbStage* d_stage, const LtbStage& h,
                              const LtbBufTable& bt, int splits, int sms,
                              cudaStream_t st) {
  int64_t outs = 1;
  for (int k = 0; k < h.nout; ++k) outs *= h.size[k];
  const int threads = h.red_total >= 256 ? 256 : 128;
  int64_t gx = outs < (int64_t)sms * 64 ? outs : (int64_t)sms * 64;
  if (gx < 1) gx = 1;
  dim3 grid((unsigned)gx, (unsigned)splits);
  k_reduce_par<<<grid, threads, 0, st>>>(d_stage, bt, outs);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || splits == 1) return e;
  k_reduce_combine<<<grid_for(outs, 256, sms), 256, 0, st>>>(d_stage, bt, outs,
                                                             splits);
  return cudaGetLastError();
}

cudaError_t ltb_launch_row_chain(const LtbStage* d_stages, int nsteps,
                                 const LtbStage& final_stage,
                                 const LtbBufTable& bt, int sms,
                                 cudaStream_t st) {
  if (nsteps > kMaxChain) return cudaErrorInvalidValue;
  int64_t rows = 1;
  for (int k = 0; k < final_stage.nout - 1; ++k) rows *= final_stage.size[k];
  const int64_t inner = final_stage.size[final_stage.nout - 1];
  const int threads = inner >= 4096 ? 512 : (inner >= 1024 ? 256 : 128);
  int64_t grid = rows < (int64_t)sms * 8 ? rows : (int64_t)sms * 8;
  if (grid < 1) grid = 1;
  k_row_chain<<<(unsigned)grid, threads, 0, st>>>(d_stages, nsteps, bt, rows);
  return cudaGetLastError();
}
