// Families (a) and (b): elementwise / broadcast / view nests and reductions,
// interpreted from LtbStage descriptors.  All of them are HBM-bound, so the
// design points are coalescing, 128-bit accesses along the innermost output
// dim, and grids sized in multiples of the 148 SMs.
#include <cfloat>
#include <map>
#include <mutex>
#include <tuple>

#include "async.cuh"
#include "compensated.cuh"
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
__device__ __forceinline__ uint32_t fdiv(uint32_t n, uint32_t mul, uint32_t shr) {
  return (__umulhi(n, mul) + n) >> shr;
}

template <int VEC>
__global__ void __launch_bounds__(256)
    k_nest(const LtbStage* __restrict__ gst, LtbBufTable bt, uint32_t nvec_mul,
           uint32_t nvec_shr) {
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
    int64_t o, iv;
    if (S.small) {  // 32-bit multiply-high division
      const uint32_t o32 = fdiv((uint32_t)w, nvec_mul, nvec_shr);
      iv = (uint32_t)w - o32 * (uint32_t)nvec;
      uint32_t r = o32;
      for (int k = ki - 1; k >= 0; --k) {
        const uint32_t q = fdiv(r, S.dm_mul[k], S.dm_shr[k]);
        x[k] = r - q * (uint32_t)S.size[k];
        r = q;
      }
      o = o32;
    } else {
      o = w / nvec;
      iv = w - o * nvec;
      int64_t r = o;
      for (int k = ki - 1; k >= 0; --k) {
        const int64_t q = r / S.size[k];
        x[k] = r - q * S.size[k];
        r = q;
      }
    }
    (void)o;
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
            for (int j = 0; j < VEC; ++j) comp_add(acc[j], comp[j], s0.v[j]);
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
    for (int j = 0; j < VEC; ++j)
      res[j] = !has_red ? s0.v[j] : S.kahan ? comp_value(acc[j], comp[j]) : acc[j];
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
        comp_add(p.v, p.c, x);
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
      // TwoSum of the running values (true sum ~= v - c)
      comp_combine(r.v, r.c, b.v, b.c);
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
        res = fold(S.red_op, S.red_init, comp_value(p.v, p.c));
      } else {
        res = comp_value(p.v, p.c);
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
      if (S.red_op == LTB_R_ADD) comp_add(acc, c, part[s]);
      else acc = fold(S.red_op, acc, part[s]);
    }
    if (S.red_op == LTB_R_ADD) acc = comp_value(acc, c);
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
            res = fold(T.red_op, T.red_init, comp_value(p.v, p.c));
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

// ---------------------------------------------------------------- linear
template <int VEC>
__device__ __forceinline__ Lanes<VEC> linear_load(const LtbLoad& L, const LtbBufTable& bt,
                                                  int64_t i0, bool full, int nv) {
  Lanes<VEC> t;
  const float* __restrict__ p = bt.p[L.buf] + L.off;
  if (L.mode == LTB_L_SCALAR) {
    const float c = __ldg(p);
#pragma unroll
    for (int j = 0; j < VEC; ++j) t.v[j] = c;
  } else if (full) {
#pragma unroll
    for (int j = 0; j < VEC; j += 4) {
      const float4 q = __ldcs(reinterpret_cast<const float4*>(p + i0 + j));
      t.v[j] = q.x; t.v[j + 1] = q.y; t.v[j + 2] = q.z; t.v[j + 3] = q.w;
    }
  } else {
#pragma unroll
    for (int j = 0; j < VEC; ++j) t.v[j] = j < nv ? p[i0 + j] : 0.f;
  }
  return t;
}

// Binary / unary maps over two (one) linear operands: the dominant
// elementwise shapes, kept small (few registers, full occupancy) with two
// 128-bit loads per operand in flight per thread.
template <int OP>
__global__ void __launch_bounds__(256)
    k_lin_bin(const float* __restrict__ a, const float* __restrict__ b, float* __restrict__ c,
              int64_t total) {
  const int64_t n8 = total / 8;
  const float4* A = reinterpret_cast<const float4*>(a);
  const float4* B = reinterpret_cast<const float4*>(b);
  float4* C = reinterpret_cast<float4*>(c);
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n8;
       v += (int64_t)gridDim.x * blockDim.x) {
    const float4 a0 = __ldcs(A + 2 * v), a1 = __ldcs(A + 2 * v + 1);
    const float4 b0 = __ldcs(B + 2 * v), b1 = __ldcs(B + 2 * v + 1);
    __stcs(C + 2 * v, make_float4(vm_bin(OP, a0.x, b0.x), vm_bin(OP, a0.y, b0.y),
                                  vm_bin(OP, a0.z, b0.z), vm_bin(OP, a0.w, b0.w)));
    __stcs(C + 2 * v + 1, make_float4(vm_bin(OP, a1.x, b1.x), vm_bin(OP, a1.y, b1.y),
                                      vm_bin(OP, a1.z, b1.z), vm_bin(OP, a1.w, b1.w)));
  }
  // ragged tail (< 8 elements)
  const int64_t t = n8 * 8 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t < total) c[t] = vm_bin(OP, a[t], b[t]);
}

template <int OP>
__global__ void __launch_bounds__(256)
    k_lin_un(const float* __restrict__ a, float* __restrict__ c, int64_t total) {
  const int64_t n8 = total / 8;
  const float4* A = reinterpret_cast<const float4*>(a);
  float4* C = reinterpret_cast<float4*>(c);
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n8;
       v += (int64_t)gridDim.x * blockDim.x) {
    const float4 a0 = __ldcs(A + 2 * v), a1 = __ldcs(A + 2 * v + 1);
    __stcs(C + 2 * v, make_float4(vm_un(OP, a0.x), vm_un(OP, a0.y), vm_un(OP, a0.z),
                                  vm_un(OP, a0.w)));
    __stcs(C + 2 * v + 1, make_float4(vm_un(OP, a1.x), vm_un(OP, a1.y), vm_un(OP, a1.z),
                                      vm_un(OP, a1.w)));
  }
  const int64_t t = n8 * 8 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t < total) c[t] = vm_un(OP, a[t]);
}

// Elementwise stages whose every load reads the output's own flat index (or
// one broadcast scalar): a pure 1-D map.  Each thread moves VEC consecutive
// floats per operand with 128-bit accesses; no index decomposition.
template <int VEC>
__global__ void __launch_bounds__(256)
    k_linear(const LtbStage* __restrict__ gst, LtbBufTable bt, int64_t total) {
  __shared__ __align__(16) LtbStage S;
  load_stage(gst, S);
  float* __restrict__ out = bt.p[S.out_buf] + S.out_off;
  bool aligned = (S.out_off & 3) == 0;
  for (int i = 0; i < S.nload; ++i)
    aligned = aligned && (S.loads[i].mode == LTB_L_SCALAR || (S.loads[i].off & 3) == 0);
  const int64_t nv_total = (total + VEC - 1) / VEC;
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nv_total;
       v += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i0 = v * VEC;
    const bool full = aligned && i0 + VEC <= total;
    const int nv = (int)(total - i0 < VEC ? total - i0 : VEC);
    // issue every operand load before the program runs: the stack moves
    // below would otherwise wait on each load in turn
    Lanes<VEC> pre[2];
#pragma unroll
    for (int li = 0; li < 2; ++li) {
      if (li < S.nload) pre[li] = linear_load<VEC>(S.loads[li], bt, i0, full, nv);
    }
    Lanes<VEC> s0{}, s1{}, s2{}, s3{}, s4{}, s5{};
    for (int i = 0; i < S.ninstr; ++i) {
      const LtbVInstr in = S.code[i];
      const int op = in.op;
      if (op == LTB_V_LOAD || op == LTB_V_CONST) {
        Lanes<VEC> t;
        if (op == LTB_V_CONST) {
#pragma unroll
          for (int j = 0; j < VEC; ++j) t.v[j] = S.consts[in.arg];
        } else if (in.arg < 2) {
          t = in.arg == 0 ? pre[0] : pre[1];
        } else {
          t = linear_load<VEC>(S.loads[in.arg], bt, i0, full, nv);
        }
        s5 = s4; s4 = s3; s3 = s2; s2 = s1; s1 = s0; s0 = t;
      } else if (op >= LTB_V_EXP) {
#pragma unroll
        for (int j = 0; j < VEC; ++j) s0.v[j] = vm_un(op, s0.v[j]);
      } else {
#pragma unroll
        for (int j = 0; j < VEC; ++j) s0.v[j] = vm_bin(op, s1.v[j], s0.v[j]);
        s1 = s2; s2 = s3; s3 = s4; s4 = s5;
      }
    }
    if (full) {
#pragma unroll
      for (int j = 0; j < VEC; j += 4)
        __stcs(reinterpret_cast<float4*>(out + i0 + j),
               make_float4(s0.v[j], s0.v[j + 1], s0.v[j + 2], s0.v[j + 3]));
    } else {
#pragma unroll
      for (int j = 0; j < VEC; ++j)
        if (j < nv) out[i0 + j] = s0.v[j];
    }
  }
}

// ---------------------------------------------------------------- window
// 8 floats from a 32-byte aligned address, streamed (evict-first): one
// whole L2 sector per thread and instruction.
__device__ __forceinline__ void ldcs_v8(const float* p, float* v) {
  asm volatile("ld.global.cs.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]),
                 "=f"(v[6]), "=f"(v[7])
               : "l"(p));
}

// Small-window reductions of one operand (pooling): out[..., o] folds
// x[... S*o + q] over q < K and the other reduced dims.  A thread makes 4
// consecutive outputs; for each outer reduced coordinate it loads the
// contiguous span of 3S+K inputs those outputs cover with 128-bit loads,
// then folds in the reference's sequential order (exact for max/min).
// U work items per thread per step (a tuned variant: 2 or 4) have all their
// span loads issued before any fold; inputs and outputs are streamed (read
// and written once, evict-first).
template <int S_, int K_, int U>
__global__ void __launch_bounds__(256)
    k_window(const LtbStage* __restrict__ gst, LtbBufTable bt, uint32_t nvec_mul,
             uint32_t nvec_shr) {
  __shared__ __align__(16) LtbStage S;
  __shared__ int64_t roff[64];
  load_stage(gst, S);
  constexpr int N = 3 * S_ + K_;
  const int no = S.nout, nd = S.ndim, ki = no - 1;
  const LtbLoad& L = S.loads[0];
  // offsets of every combination of the outer reduced dims
  const int64_t RC = S.red_total / K_;
  for (int64_t rc = threadIdx.x; rc < RC; rc += blockDim.x) {
    int64_t r = rc, o = 0;
    for (int k = nd - 2; k >= no; --k) {
      const int64_t q = r / S.size[k];
      o += L.coef[k] * (r - q * S.size[k]);
      r = q;
    }
    roff[rc] = o;
  }
  __syncthreads();
  const uint32_t inner = (uint32_t)S.size[ki];
  const uint32_t nvec = (inner + 3) / 4;
  uint32_t outer = 1;
  for (int k = 0; k < ki; ++k) outer *= (uint32_t)S.size[k];
  const uint32_t total = outer * nvec;
  const float* __restrict__ src = bt.p[L.buf];
  float* __restrict__ out = bt.p[S.out_buf];
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t w0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w0 < total;
       w0 += U * stride) {
    int64_t base[U], obase[U];
    int nv[U];
    bool live[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const uint64_t w = w0 + u * stride;
      live[u] = w < total;
      const uint32_t ww = (uint32_t)(live[u] ? w : w0);  // < total < 2^32
      const uint32_t o32 = fdiv(ww, nvec_mul, nvec_shr);
      const uint32_t iv = ww - o32 * nvec;
      int64_t b = L.off, ob = S.out_off;
      uint32_t r = o32;
      for (int k = ki - 1; k >= 0; --k) {
        const uint32_t q = fdiv(r, S.dm_mul[k], S.dm_shr[k]);
        const int64_t c = r - q * (uint32_t)S.size[k];
        b += L.coef[k] * c;
        ob += S.out_coef[k] * c;
        r = q;
      }
      const int64_t o0 = (int64_t)iv * 4;
      base[u] = b + L.coef[ki] * o0;
      obase[u] = ob + o0;
      nv[u] = (int)(inner - o0 < 4 ? inner - o0 : 4);
    }
    float acc[U][4];
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[u][j] = S.red_init;
#pragma unroll 2
    for (int64_t rc = 0; rc < RC; ++rc) {
      float span[U][N];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const float* p = src + base[u] + roff[rc];
        if (N % 8 == 0 && nv[u] == 4 && (reinterpret_cast<uintptr_t>(p) & 31) == 0) {
          // whole 32-byte sectors: one load per sector, so a warp's
          // neighbouring spans do not each take half of the same sectors
#pragma unroll
          for (int q = 0; q + 8 <= N; q += 8) ldcs_v8(p + q, &span[u][q]);
        } else if (nv[u] == 4 && ((base[u] + roff[rc]) & 3) == 0) {
#pragma unroll
          for (int q = 0; q + 4 <= N; q += 4) {
            const float4 t = __ldcs(reinterpret_cast<const float4*>(p + q));
            span[u][q] = t.x; span[u][q + 1] = t.y; span[u][q + 2] = t.z; span[u][q + 3] = t.w;
          }
#pragma unroll
          for (int q = N & ~3; q < N; ++q) span[u][q] = __ldcs(p + q);
        } else {
#pragma unroll
          for (int q = 0; q < N; ++q)
            span[u][q] = q <= (nv[u] - 1) * S_ + K_ - 1 ? __ldcs(p + q) : 0.f;
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u)
#pragma unroll
        for (int q = 0; q < K_; ++q)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[u][j] = fold(S.red_op, acc[u][j], span[u][j * S_ + q]);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (!live[u]) continue;
      float* o = out + obase[u];
      if (nv[u] == 4 && (obase[u] & 3) == 0) {
        __stcs(reinterpret_cast<float4*>(o),
               make_float4(acc[u][0], acc[u][1], acc[u][2], acc[u][3]));
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (j < nv[u]) o[j] = acc[u][j];
      }
    }
  }
}

// ----------------------------------------------------------- row softmax
// Fused pattern m = max_n x, s = sum_n exp(x - m), y = exp(x - m) / s
// (computed as e * (1/s) with a correctly rounded reciprocal), the
// row held in registers (EPT floats per thread, loaded and stored as
// float4), so HBM sees one read and one write per element.  One full wave
// of CTAs strides over the rows; while a row is reduced the next row's loads
// are already in flight (register double buffer).  The addressing of the
// chain's three stages is flattened on the host into one parameter block.
// The max is the reference's ternary fold from -FLT_MAX; its tie and NaN
// order cannot change y (a NaN anywhere makes s, hence every y, NaN).
struct SoftmaxRows {
  const float* x;
  float *y, *m, *s;
  int64_t xoff, yoff, moff, soff, n, rows;
  int nd;  // row dims
  int64_t size[LTB_MAXD], xc[LTB_MAXD], yc[LTB_MAXD], mc[LTB_MAXD], sc[LTB_MAXD];
};

struct RowOffs {
  int64_t x, y, m, s;
};

__device__ __forceinline__ RowOffs row_offs(const SoftmaxRows& P, int64_t row) {
  RowOffs o{P.xoff, P.yoff, P.moff, P.soff};
  for (int k = P.nd - 1; k >= 0; --k) {
    const int64_t q = k ? row / P.size[k] : 0;
    const int64_t c = row - q * P.size[k];
    row = q;
    o.x += P.xc[k] * c;
    o.y += P.yc[k] * c;
    o.m += P.mc[k] * c;
    o.s += P.sc[k] * c;
  }
  return o;
}

template <int EPT, int NT>
__device__ __forceinline__ void softmax_load(const SoftmaxRows& P, int64_t xoff, bool v4,
                                             float (&v)[EPT]) {
#pragma unroll
  for (int q = 0; q < EPT / 4; ++q) {
    const int64_t j = (int64_t)(q * NT + threadIdx.x) * 4;
    if (v4 && j < P.n) {
      const float4 t = __ldcs(reinterpret_cast<const float4*>(P.x + xoff + j));
      v[4 * q] = t.x; v[4 * q + 1] = t.y; v[4 * q + 2] = t.z; v[4 * q + 3] = t.w;
    } else {
#pragma unroll
      for (int e = 0; e < 4; ++e) v[4 * q + e] = j + e < P.n ? P.x[xoff + j + e] : -INFINITY;
    }
  }
}

template <int EPT, int NT>
__global__ void __launch_bounds__(NT)
    k_softmax_rows(const __grid_constant__ SoftmaxRows P) {
  __shared__ float red[2][NT / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int64_t row = blockIdx.x;
  if (row >= P.rows) return;
  const bool vec_ok = (P.n & 3) == 0;
  float v[EPT], nx[EPT];
  RowOffs o = row_offs(P, row);
  bool v4 = vec_ok && ((o.x | o.y) & 3) == 0;
  softmax_load<EPT, NT>(P, o.x, v4, v);
  for (; row < P.rows; row += gridDim.x) {
    const int64_t nrow = row + gridDim.x;
    RowOffs no = o;
    bool nv4 = v4;
    if (nrow < P.rows) {  // next row's loads go out before this row's reductions
      no = row_offs(P, nrow);
      nv4 = vec_ok && ((no.x | no.y) & 3) == 0;
      softmax_load<EPT, NT>(P, no.x, nv4, nx);
    }
    float m = -FLT_MAX;
#pragma unroll
    for (int e = 0; e < EPT; ++e) m = m > v[e] ? m : v[e];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const float t = __shfl_xor_sync(0xffffffffu, m, off);
      m = m > t ? m : t;
    }
    if (lane == 0) red[0][wid] = m;
    __syncthreads();
    m = red[0][0];
#pragma unroll
    for (int w = 1; w < NT / 32; ++w) m = m > red[0][w] ? m : red[0][w];
    float sum = 0.f;
#pragma unroll
    for (int e = 0; e < EPT; ++e) {
      v[e] = expf(v[e] - m);
      sum += v[e];
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, off);
    if (lane == 0) red[1][wid] = sum;
    __syncthreads();
    sum = 0.f;
#pragma unroll
    for (int w = 0; w < NT / 32; ++w) sum += red[1][w];
    if (threadIdx.x == 0) {  // per-row results stay visible to later stages
      P.m[o.m] = m;
      P.s[o.s] = sum;
    }
    // y = e * (1 / s): one correctly rounded reciprocal per row, within
    // 1.5 ulp of e / s
    const float inv = __frcp_rn(sum);
#pragma unroll
    for (int q = 0; q < EPT / 4; ++q) {
      const int64_t j = (int64_t)(q * NT + threadIdx.x) * 4;
      if (v4 && j < P.n) {
        __stcs(reinterpret_cast<float4*>(P.y + o.y + j),
               make_float4(v[4 * q] * inv, v[4 * q + 1] * inv, v[4 * q + 2] * inv,
                           v[4 * q + 3] * inv));
      } else {
#pragma unroll
        for (int e = 0; e < 4; ++e)
          if (j + e < P.n) P.y[o.y + j + e] = v[4 * q + e] * inv;
      }
    }
#pragma unroll
    for (int e = 0; e < EPT; ++e) v[e] = nx[e];
    o = no;
    v4 = nv4;
  }
}

// TMA-staged form: each CTA keeps kSmxRing of its rows in flight in a
// shared-memory ring, one 1-D bulk copy (cp.async.bulk) per row completing
// on the slot's mbarrier; a slot is refilled with the row kSmxRing ahead as
// soon as every thread has read it.  Needs 16-byte aligned rows.  Same
// arithmetic as k_softmax_rows.  A copy that does not land within the
// bounded wait raises *err; the CTA then waits (bounded) for the copies it
// still has in flight and exits.
constexpr int kSmxRing = 4;

template <int EPT, int NT>
__global__ void __launch_bounds__(NT)
    k_softmax_bulk(const __grid_constant__ SoftmaxRows P, int* err) {
  extern __shared__ __align__(128) float ring[];  // kSmxRing x n floats
  __shared__ __align__(8) uint64_t bars[kSmxRing];
  __shared__ float red[2][NT / 32];
  __shared__ int stop;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int64_t first = blockIdx.x;
  if (first >= P.rows) return;
  const int64_t cnt = (P.rows - first + gridDim.x - 1) / gridDim.x;  // rows of this CTA
  const uint32_t bytes = (uint32_t)(P.n * 4);
  if (threadIdx.x == 0) {
    for (int s = 0; s < kSmxRing; ++s) mbar_init(smem_u32(&bars[s]), 1);
    fence_mbar_init();
    stop = 0;
  }
  __syncthreads();
  auto issue = [&](int64_t i) {  // row i of this CTA into slot i % kSmxRing
    const int s = (int)(i % kSmxRing);
    const RowOffs o = row_offs(P, first + i * gridDim.x);
    const uint32_t bar = smem_u32(&bars[s]);
    mbar_expect_tx(bar, bytes);
    bulk_load(smem_u32(ring + (size_t)s * P.n), P.x + o.x, bytes, bar);
  };
  if (threadIdx.x == 0)
    for (int64_t i = 0; i < cnt && i < kSmxRing; ++i) issue(i);
  int64_t i = 0;
  for (; i < cnt; ++i) {
    const int s = (int)(i % kSmxRing);
    if (!mbar_wait(smem_u32(&bars[s]), (uint32_t)((i / kSmxRing) & 1), err)) stop = 1;
    __syncthreads();
    if (stop) break;
    const RowOffs o = row_offs(P, first + i * gridDim.x);
    const float* xs = ring + (size_t)s * P.n;
    float v[EPT];
#pragma unroll
    for (int q = 0; q < EPT / 4; ++q) {
      const int64_t j = (int64_t)(q * NT + threadIdx.x) * 4;
      if (j < P.n) {
        const float4 t = *reinterpret_cast<const float4*>(xs + j);
        v[4 * q] = t.x; v[4 * q + 1] = t.y; v[4 * q + 2] = t.z; v[4 * q + 3] = t.w;
      } else {
        v[4 * q] = v[4 * q + 1] = v[4 * q + 2] = v[4 * q + 3] = -INFINITY;
      }
    }
    float m = -FLT_MAX;
#pragma unroll
    for (int e = 0; e < EPT; ++e) m = m > v[e] ? m : v[e];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const float t = __shfl_xor_sync(0xffffffffu, m, off);
      m = m > t ? m : t;
    }
    if (lane == 0) red[0][wid] = m;
    __syncthreads();  // every thread has read slot s: refill it
    if (threadIdx.x == 0 && i + kSmxRing < cnt) issue(i + kSmxRing);
    m = red[0][0];
#pragma unroll
    for (int w = 1; w < NT / 32; ++w) m = m > red[0][w] ? m : red[0][w];
    float sum = 0.f;
#pragma unroll
    for (int e = 0; e < EPT; ++e) {
      v[e] = expf(v[e] - m);
      sum += v[e];
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, off);
    if (lane == 0) red[1][wid] = sum;
    __syncthreads();
    sum = 0.f;
#pragma unroll
    for (int w = 0; w < NT / 32; ++w) sum += red[1][w];
    if (threadIdx.x == 0) {
      P.m[o.m] = m;
      P.s[o.s] = sum;
    }
    // y = e * (1 / s): one correctly rounded reciprocal per row, within
    // 1.5 ulp of e / s
    const float inv = __frcp_rn(sum);
    const bool v4 = (o.y & 3) == 0;
#pragma unroll
    for (int q = 0; q < EPT / 4; ++q) {
      const int64_t j = (int64_t)(q * NT + threadIdx.x) * 4;
      if (v4 && j < P.n) {
        __stcs(reinterpret_cast<float4*>(P.y + o.y + j),
               make_float4(v[4 * q] * inv, v[4 * q + 1] * inv, v[4 * q + 2] * inv,
                           v[4 * q + 3] * inv));
      } else {
#pragma unroll
        for (int e = 0; e < 4; ++e)
          if (j + e < P.n) P.y[o.y + j + e] = v[4 * q + e] * inv;
      }
    }
  }
  // stopped early: rows [i, i + kSmxRing) may still be landing
  if (threadIdx.x == 0 && i < cnt)
    for (int64_t k = i; k < cnt && k < i + kSmxRing; ++k)
      mbar_drain(smem_u32(&bars[k % kSmxRing]), (uint32_t)((k / kSmxRing) & 1));
}

}  // namespace

// ------------------------------------------------------------ launchers
// Resident CTAs per SM of a kernel at a block size (occupancy calculator,
// cached per kernel and block size).  By default grid-stride kernels launch
// exactly one full wave (SMs x resident CTAs); a schedule's cta_per_sm
// overrides that (more CTAs than resident = several waves).
static int resident(const void* kernel, int threads, size_t smem = 0) {
  static std::mutex mu;
  static std::map<std::tuple<const void*, int, size_t>, int> cache;
  const auto key = std::make_tuple(kernel, threads, smem);
  std::lock_guard<std::mutex> g(mu);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, smem) != cudaSuccess ||
      n < 1) {
    cudaGetLastError();
    n = 1;
  }
  cache[key] = n;
  return n;
}

template <typename K>
static int grid_of(K kernel, int64_t work, int threads, int sms, const LtbCfg& cfg,
                   size_t smem = 0) {
  if (cfg.grid > 0) return cfg.grid;  // pinned (grid-stride kernels cover any work)
  int64_t blocks = (work + threads - 1) / threads;
  const int per_sm = cfg.cta_per_sm > 0
                         ? cfg.cta_per_sm
                         : resident(reinterpret_cast<const void*>(kernel), threads, smem);
  const int64_t cap = (int64_t)sms * per_sm;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  return (int)blocks;
}

static int pick_threads(const LtbCfg& cfg, int dflt, int maxt) {
  const int t = cfg.threads > 0 ? cfg.threads : dflt;
  return t > maxt ? maxt : t;
}

static const int kWaves[] = {0, 1, 2, 4, 8, 16, 32};

cudaError_t ltb_smem_optin(const void* fn, size_t bytes) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, size_t> done;  // (kernel, device) -> bytes
  std::lock_guard<std::mutex> g(mu);
  size_t& have = done[{fn, dev}];
  if (have >= bytes) return cudaSuccess;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) have = bytes;
  return e;
}

// Pooling-shaped reductions (k_window): one operand, unit-stride innermost
// window, at most 64 outer window positions; *s = output stride, *k =
// innermost window extent.
static bool window_shape(const LtbStage& h, int64_t* s, int64_t* k) {
  const LtbLoad& L0 = h.loads[0];
  if (!(h.small && h.nout >= 1 && h.ndim > h.nout && h.nload == 1 && h.ninstr == 2 &&
        h.code[0].op == LTB_V_LOAD && h.code[1].op == LTB_V_FOLD && L0.nq == 0 && L0.ng == 0 &&
        h.out_coef[h.nout - 1] == 1 && L0.coef[h.ndim - 1] == 1 &&
        h.red_total / h.size[h.ndim - 1] <= 64 && h.red_op != LTB_R_SUB &&
        h.red_op != LTB_R_DIV && !h.kahan))
    return false;
  *s = L0.coef[h.nout - 1];
  *k = h.size[h.ndim - 1];
  return true;
}

int ltb_nest_candidates(const LtbStage& h, LtbCfg* out, int cap) {
  int n = 0;
  int64_t s = 0, k = 0;
  const bool win = !h.linear && h.nout >= 1 && h.size[h.nout - 1] >= 4 && window_shape(h, &s, &k);
  for (int w : kWaves)
    for (int t : {128, 256})
      for (int v : {0, 4})  // pooling: 2 or 4 work items per thread
        if (n < cap && (v == 0 || win)) out[n++] = LtbCfg{w, t, v};
  return n;
}

int ltb_reduce_candidates(const LtbStage& h, LtbCfg* out, int cap) {
  int n = 0;
  for (int w : {0, 2, 4, 8, 16, 64})
    for (int t : {64, 128, 256})
      if (n < cap && (t <= 128 || h.red_total >= 256)) out[n++] = LtbCfg{w, t, 0};
  return n;
}

cudaError_t ltb_launch_nest(const LtbStage* d_stage, const LtbStage& h,
                            const LtbBufTable& bt, int sms, cudaStream_t st,
                            const LtbCfg& cfg) {
  const int no = h.nout;
  const int64_t inner = no ? h.size[no - 1] : 1;
  int64_t outer = 1;
  for (int k = 0; k < no - 1; ++k) outer *= h.size[k];
  const int threads = pick_threads(cfg, 256, 256);
  if (h.linear) {
    int64_t total = outer * inner;
    const int64_t work8 = (total + 7) / 8;
    // [LOAD a, LOAD b, op] / [LOAD a, op] over linear, 16B-aligned operands
    auto lin = [&](int i) {
      const LtbLoad& L = h.loads[h.code[i].arg];
      return L.mode == LTB_L_LINEAR && (L.off & 3) == 0;
    };
    float* out = bt.p[h.out_buf] + h.out_off;
    if (total >= 8 && (h.out_off & 3) == 0 && h.ninstr == 3 && h.code[0].op == LTB_V_LOAD &&
        h.code[1].op == LTB_V_LOAD && lin(0) && lin(1) && h.code[2].op >= LTB_V_ADD &&
        h.code[2].op <= LTB_V_MAX) {
      const float* a = bt.p[h.loads[h.code[0].arg].buf] + h.loads[h.code[0].arg].off;
      const float* b = bt.p[h.loads[h.code[1].arg].buf] + h.loads[h.code[1].arg].off;
      switch (h.code[2].op) {
#define LTB_BIN(O)                                                                  \
  case O:                                                                           \
    k_lin_bin<O><<<grid_of(k_lin_bin<O>, work8, threads, sms, cfg), threads, 0, st>>>( \
        a, b, out, total);                                                          \
    break;
        LTB_BIN(LTB_V_ADD) LTB_BIN(LTB_V_SUB) LTB_BIN(LTB_V_MUL) LTB_BIN(LTB_V_DIV)
        LTB_BIN(LTB_V_MIN) LTB_BIN(LTB_V_MAX)
#undef LTB_BIN
      }
      return cudaGetLastError();
    }
    if (total >= 8 && (h.out_off & 3) == 0 && h.ninstr == 2 && h.code[0].op == LTB_V_LOAD &&
        lin(0) && h.code[1].op >= LTB_V_EXP && h.code[1].op <= LTB_V_RECIP) {
      const float* a = bt.p[h.loads[h.code[0].arg].buf] + h.loads[h.code[0].arg].off;
      switch (h.code[1].op) {
#define LTB_UN(O)                                                                 \
  case O:                                                                         \
    k_lin_un<O><<<grid_of(k_lin_un<O>, work8, threads, sms, cfg), threads, 0, st>>>( \
        a, out, total);                                                           \
    break;
        LTB_UN(LTB_V_EXP) LTB_UN(LTB_V_LOG) LTB_UN(LTB_V_SQRT) LTB_UN(LTB_V_ABS)
        LTB_UN(LTB_V_NEG) LTB_UN(LTB_V_RECIP)
#undef LTB_UN
      }
      return cudaGetLastError();
    }
    k_linear<4><<<grid_of(k_linear<4>, (total + 3) / 4, threads, sms, cfg), threads, 0, st>>>(
        d_stage, bt, total);
    return cudaGetLastError();
  }
  const bool vec = inner >= 4;
  const int64_t nvec = vec ? (inner + 3) / 4 : inner;
  const int64_t work = outer * nvec;
  uint32_t l = 0;
  while (l < 32 && (int64_t(1) << l) < nvec) ++l;
  const uint32_t mul =
      (uint32_t)((((uint64_t(1) << 32) * ((uint64_t(1) << l) - (uint64_t)nvec)) / (uint64_t)nvec) + 1);
  int64_t s = 0, k = 0;
  if (vec && window_shape(h, &s, &k)) {
#define LTB_WIN(SS, KK)                                                                   \
  if (s == SS && k == KK) {                                                               \
    if (cfg.variant == 4)                                                                 \
      k_window<SS, KK, 4><<<grid_of(k_window<SS, KK, 4>, work, threads, sms, cfg), threads, \
                            0, st>>>(d_stage, bt, mul, l);                                \
    else                                                                                  \
      k_window<SS, KK, 2><<<grid_of(k_window<SS, KK, 2>, work, threads, sms, cfg), threads, \
                            0, st>>>(d_stage, bt, mul, l);                                \
    return cudaGetLastError();                                                            \
  }
    LTB_WIN(2, 2) LTB_WIN(1, 2) LTB_WIN(1, 3) LTB_WIN(2, 3) LTB_WIN(3, 3) LTB_WIN(1, 1)
    LTB_WIN(2, 1)
#undef LTB_WIN
  }
  if (vec)
    k_nest<4><<<grid_of(k_nest<4>, work, threads, sms, cfg), threads, 0, st>>>(d_stage, bt, mul,
                                                                                l);
  else
    k_nest<1><<<grid_of(k_nest<1>, work, threads, sms, cfg), threads, 0, st>>>(d_stage, bt, mul,
                                                                                l);
  return cudaGetLastError();
}

// The plain linear maps (k_lin_bin / k_lin_un patterns): every load reads
// the output's own flat index, so any flat sub-range runs on its own.
static bool linear_map(const LtbStage& h, int* nload) {
  if (!h.linear || (h.out_off & 3)) return false;
  auto lin = [&](int i) {
    const LtbLoad& L = h.loads[h.code[i].arg];
    return L.mode == LTB_L_LINEAR && (L.off & 3) == 0;
  };
  if (h.ninstr == 3 && h.code[0].op == LTB_V_LOAD && h.code[1].op == LTB_V_LOAD && lin(0) &&
      lin(1) && h.code[2].op >= LTB_V_ADD && h.code[2].op <= LTB_V_MAX) {
    *nload = 2;
    return true;
  }
  if (h.ninstr == 2 && h.code[0].op == LTB_V_LOAD && lin(0) && h.code[1].op >= LTB_V_EXP &&
      h.code[1].op <= LTB_V_RECIP) {
    *nload = 1;
    return true;
  }
  return false;
}

int ltb_linear_range_ok(const LtbStage& h) {
  int nl = 0;
  if (!linear_map(h, &nl) || h.out_off) return 0;
  for (int i = 0; i < nl; ++i)
    if (h.loads[h.code[i].arg].off) return 0;  // element e of every buffer is flat index e
  return 1;
}

cudaError_t ltb_launch_linear_range(const LtbStage& h, const LtbBufTable& bt, int64_t lo,
                                    int64_t n, int sms, cudaStream_t st, const LtbCfg& cfg) {
  int nl = 0;
  if (!linear_map(h, &nl) || (lo & 7) || n <= 0) return cudaErrorNotSupported;
  const int threads = pick_threads(cfg, 256, 256);
  const int64_t work8 = (n + 7) / 8;
  float* out = bt.p[h.out_buf] + h.out_off + lo;
  const LtbLoad& L0 = h.loads[h.code[0].arg];
  const float* a = bt.p[L0.buf] + L0.off + lo;
  if (nl == 2) {
    const LtbLoad& L1 = h.loads[h.code[1].arg];
    const float* b = bt.p[L1.buf] + L1.off + lo;
    switch (h.code[2].op) {
#define LTB_BIN(O)                                                                  \
  case O:                                                                           \
    k_lin_bin<O><<<grid_of(k_lin_bin<O>, work8, threads, sms, cfg), threads, 0, st>>>( \
        a, b, out, n);                                                              \
    break;
      LTB_BIN(LTB_V_ADD) LTB_BIN(LTB_V_SUB) LTB_BIN(LTB_V_MUL) LTB_BIN(LTB_V_DIV)
      LTB_BIN(LTB_V_MIN) LTB_BIN(LTB_V_MAX)
#undef LTB_BIN
    }
  } else {
    switch (h.code[1].op) {
#define LTB_UN(O)                                                                 \
  case O:                                                                         \
    k_lin_un<O><<<grid_of(k_lin_un<O>, work8, threads, sms, cfg), threads, 0, st>>>( \
        a, out, n);                                                               \
    break;
      LTB_UN(LTB_V_EXP) LTB_UN(LTB_V_LOG) LTB_UN(LTB_V_SQRT) LTB_UN(LTB_V_ABS)
      LTB_UN(LTB_V_NEG) LTB_UN(LTB_V_RECIP)
#undef LTB_UN
    }
  }
  return cudaGetLastError();
}

cudaError_t ltb_launch_reduce(const LtbStage* d_stage, const LtbStage& h,
                              const LtbBufTable& bt, int splits, int sms,
                              cudaStream_t st, const LtbCfg& cfg) {
  int64_t outs = 1;
  for (int k = 0; k < h.nout; ++k) outs *= h.size[k];
  const int threads = pick_threads(cfg, h.red_total >= 256 ? 256 : 128, 256);
  // one CTA per output, up to a cap of CTAs per SM (block-stride over outputs)
  const int64_t per_sm = cfg.cta_per_sm > 0 ? cfg.cta_per_sm : 64;
  int64_t gx = outs < (int64_t)sms * per_sm ? outs : (int64_t)sms * per_sm;
  if (cfg.grid > 0) gx = cfg.grid < outs ? cfg.grid : outs;  // pinned
  if (gx < 1) gx = 1;
  dim3 grid((unsigned)gx, (unsigned)splits);
  k_reduce_par<<<grid, threads, 0, st>>>(d_stage, bt, outs);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || splits == 1) return e;
  k_reduce_combine<<<grid_of(k_reduce_combine, outs, 256, sms, LtbCfg{0, 0, 0}), 256, 0, st>>>(
      d_stage, bt, outs, splits);
  return cudaGetLastError();
}

// Row-softmax schedules: (elements per thread, threads) pairs covering the
// row; variant v (1-based) indexes this table.  Variants 1-11 hold the next
// row in registers (k_softmax_rows), 12-17 stage rows through a shared
// memory ring with bulk copies (k_softmax_bulk).
static const int kSmxVariants[][2] = {{4, 128},  {4, 256},  {8, 256},  {16, 256},
                                      {32, 256}, {8, 128},  {16, 128}, {32, 128},
                                      {4, 512},  {8, 512},  {16, 512}, {4, 256},
                                      {8, 256},  {16, 256}, {32, 256}, {8, 512},
                                      {16, 512}};
constexpr int kFirstBulk = 12;
constexpr int kNumSmx = sizeof(kSmxVariants) / sizeof(kSmxVariants[0]);

static bool softmax_chain(const LtbStage* const* h_stages, int nsteps) {
  const LtbStage& f = *h_stages[nsteps - 1];
  return f.pattern == LTB_P_SOFTMAX && nsteps == 3 && f.size[f.nout - 1] <= 256 * 32;
}

// heuristic variant: the smallest EPT x 256 that covers the row
static int softmax_default(int64_t inner) {
  if (inner <= 128 * 4) return 1;
  if (inner <= 256 * 4) return 2;
  if (inner <= 256 * 8) return 3;
  if (inner <= 256 * 16) return 4;
  return 5;
}

static bool softmax_fits(int v, int64_t inner) {
  const int e = kSmxVariants[v - 1][0], t = kSmxVariants[v - 1][1];
  return (int64_t)e * t >= inner && ((int64_t)e * t <= 2 * inner || e == 4);
}

// Rows staged by bulk copies must start on 16-byte boundaries (x offsets
// and row strides multiples of 4 floats) and a ring of kSmxRing rows must
// fit in shared memory.
static bool softmax_bulk_ok(const LtbStage* const* h_stages, int nsteps) {
  const LtbStage& A = *h_stages[0];
  const LtbStage& C = *h_stages[nsteps - 1];
  const LtbLoad& X = A.loads[A.code[0].arg];
  const int64_t n = C.size[C.nout - 1];
  if ((n & 3) || (X.off & 3) || n * 4 * kSmxRing > 200 * 1024) return false;
  for (int k = 0; k < C.nout - 1; ++k)
    if (X.coef[k] & 3) return false;
  return true;
}

int ltb_row_chain_candidates(const LtbStage* const* h_stages, int nsteps, LtbCfg* out, int cap) {
  int n = 0;
  if (softmax_chain(h_stages, nsteps)) {
    const LtbStage& f = *h_stages[nsteps - 1];
    const int64_t inner = f.size[f.nout - 1];
    const bool bulk = softmax_bulk_ok(h_stages, nsteps);
    for (int v = 1; v <= kNumSmx; ++v)
      if (softmax_fits(v, inner) && (v < kFirstBulk || bulk))
        for (int w : {0, 2, 4, 8})
          if (n < cap) out[n++] = LtbCfg{w, 0, v};
    return n;
  }
  for (int w : {0, 2, 4, 8, 16})
    for (int t : {128, 256, 512})
      if (n < cap) out[n++] = LtbCfg{w, t, 0};
  return n;
}

template <int EPT, int NT>
static cudaError_t launch_softmax_bulk(const SoftmaxRows& P, int sms, const LtbCfg& cfg,
                                       int* err, cudaStream_t st) {
  const size_t smem = (size_t)kSmxRing * P.n * 4;
  {
    const cudaError_t e = ltb_smem_optin((const void*)k_softmax_bulk<EPT, NT>, smem);
    if (e != cudaSuccess) return e;
  }
  const int g = grid_of(k_softmax_bulk<EPT, NT>, P.rows * NT, NT, sms, cfg, smem);
  k_softmax_bulk<EPT, NT><<<g, NT, smem, st>>>(P, err);
  return cudaGetLastError();
}

cudaError_t ltb_launch_row_chain(const LtbStage* d_stages, const LtbStage* const* h_stages,
                                 int nsteps, const LtbBufTable& bt, int sms,
                                 cudaStream_t st, const LtbCfg& cfg, int* err) {
  if (nsteps > kMaxChain) return cudaErrorInvalidValue;
  const LtbStage& final_stage = *h_stages[nsteps - 1];
  int64_t rows = 1;
  for (int k = 0; k < final_stage.nout - 1; ++k) rows *= final_stage.size[k];
  const int64_t inner = final_stage.size[final_stage.nout - 1];
  if (softmax_chain(h_stages, nsteps)) {
    const LtbStage& A = *h_stages[0];  // max over n
    const LtbStage& B = *h_stages[1];  // sum over n
    const LtbStage& C = final_stage;   // elementwise output
    const LtbLoad& X = A.loads[A.code[0].arg];
    SoftmaxRows P{};
    P.x = bt.p[X.buf];
    P.y = bt.p[C.out_buf];
    P.m = bt.p[A.out_buf];
    P.s = bt.p[B.out_buf];
    P.xoff = X.off;
    P.yoff = C.out_off;
    P.moff = A.out_off;
    P.soff = B.out_off;
    P.n = inner;
    P.rows = rows;
    P.nd = C.nout - 1;
    for (int k = 0; k < P.nd; ++k) {
      P.size[k] = C.size[k];
      P.xc[k] = X.coef[k];
      P.yc[k] = C.out_coef[k];
      P.mc[k] = A.out_coef[k];
      P.sc[k] = B.out_coef[k];
    }
    int v = cfg.variant;
    const bool bulk = softmax_bulk_ok(h_stages, nsteps) &&
                      (reinterpret_cast<uintptr_t>(P.x) & 15) == 0;
    if (v < 1 || v > kNumSmx || !softmax_fits(v, inner) || (v >= kFirstBulk && !bulk))
      v = softmax_default(inner);
    switch (v) {
#define LTB_SMX(V, EPT, NT)                                                            \
  case V: {                                                                            \
    const int g = grid_of(k_softmax_rows<EPT, NT>, rows * NT, NT, sms, cfg);           \
    k_softmax_rows<EPT, NT><<<g, NT, 0, st>>>(P);                                      \
    return cudaGetLastError();                                                         \
  }
      LTB_SMX(1, 4, 128) LTB_SMX(2, 4, 256) LTB_SMX(3, 8, 256) LTB_SMX(4, 16, 256)
      LTB_SMX(5, 32, 256) LTB_SMX(6, 8, 128) LTB_SMX(7, 16, 128) LTB_SMX(8, 32, 128)
      LTB_SMX(9, 4, 512) LTB_SMX(10, 8, 512) LTB_SMX(11, 16, 512)
#undef LTB_SMX
      case 12: return launch_softmax_bulk<4, 256>(P, sms, cfg, err, st);
      case 13: return launch_softmax_bulk<8, 256>(P, sms, cfg, err, st);
      case 14: return launch_softmax_bulk<16, 256>(P, sms, cfg, err, st);
      case 15: return launch_softmax_bulk<32, 256>(P, sms, cfg, err, st);
      case 16: return launch_softmax_bulk<8, 512>(P, sms, cfg, err, st);
      case 17: return launch_softmax_bulk<16, 512>(P, sms, cfg, err, st);
    }
    return cudaErrorInvalidValue;
  }
  const int threads =
      pick_threads(cfg, inner >= 4096 ? 512 : (inner >= 1024 ? 256 : 128), 512);
  const int64_t per_sm = cfg.cta_per_sm > 0 ? cfg.cta_per_sm : 8;
  int64_t grid = rows < (int64_t)sms * per_sm ? rows : (int64_t)sms * per_sm;
  if (grid < 1) grid = 1;
  k_row_chain<<<(unsigned)grid, threads, 0, st>>>(d_stages, nsteps, bt, rows);
  return cudaGetLastError();
}
