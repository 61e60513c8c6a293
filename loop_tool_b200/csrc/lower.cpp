#include "lower.hpp"

#include <algorithm>
#include <cfloat>
#include <cstring>
#include <functional>
#include <map>
#include <set>
#include <sstream>

namespace ltb {

const char* family_name(Family f) {
  switch (f) {
    case Family::elementwise: return "elementwise";
    case Family::reduce_serial: return "reduce_serial";
    case Family::reduce_parallel: return "reduce_parallel";
    case Family::reduce_split: return "reduce_split";
    case Family::row_chain: return "row_chain";
    case Family::contraction: return "contraction";
  }
  return "?";
}

namespace {

bool is_compute(Op op) {
  return op != Op::read && op != Op::write && op != Op::view &&
         op != Op::constant && op != Op::name;
}
bool is_unary(Op op) {
  return op == Op::exp || op == Op::log || op == Op::sqrt || op == Op::abs ||
         op == Op::negate || op == Op::reciprocal;
}
bool contains(const std::vector<int>& v, int x) {
  return std::find(v.begin(), v.end(), x) != v.end();
}

struct Access {
  int base = -1;
  std::vector<ExP> idx;  // one expression per var of the base node
  bool through_view = false;
};

// Restatement of Compiler::gen_index_equations' get_expr (compile.cpp:
// 634-692) in the read direction: the expression for `var` (a var of the
// view's input) in terms of the view's output vars.
ExP view_expr(const IRGraph& g, int view, int var) {
  const Node& V = g.nodes[view];
  auto is_out = [&](int v) { return contains(V.vars, v); };
  for (const auto& c : V.constraints) {
    if (!(c.lhs->op == EOp::var && c.lhs->var == var)) continue;
    std::vector<int> syms;
    ex_vars(c.rhs, syms, false);
    bool only_out = std::all_of(syms.begin(), syms.end(), is_out);
    if (only_out) return c.rhs;
    // bijective views: drop non-output vars, wrapping in a modulus by
    // their (negated) stride
    if (!g.view_has_reduction(view)) {
      ExP e = c.rhs;
      for (int s : syms) {
        if (is_out(s)) continue;
        ExP mod = ex_un(EOp::negate, ex_diff(e, s));
        e = ex_simplify(ex_replace_var(e, s, ex_val(0)));
        float mf;
        if (ex_eval_float(mod, &mf) && mf > 1)
          e = ex_bin(EOp::modulo, e, ex_simplify(mod));
      }
      std::vector<int> rest;
      ex_vars(e, rest, false);
      if (std::all_of(rest.begin(), rest.end(), is_out)) return e;
    }
  }
  return ex_var(var);
}

// Index expressions with which `consumer` reads `input` (compile.cpp:
// 611-756 collect_fw): walk the view chain from the base upward,
// substituting every base-side var that is not directly available at the
// consumer.
Access derive_access(const IRGraph& g, int consumer, int input) {
  Access acc;
  std::vector<int> chain;  // consumer side first
  int x = input;
  while (g.nodes[x].op == Op::view) {
    LTB_CHECK(g.nodes[x].inputs.size() == 1, "view must have one input");
    chain.push_back(x);
    x = g.nodes[x].inputs[0];
  }
  acc.base = x;
  acc.through_view = !chain.empty();
  for (int v : g.nodes[x].vars) acc.idx.push_back(ex_var(v));
  auto avail = g.all_vars(consumer);
  for (auto it = chain.rbegin(); it != chain.rend(); ++it) {
    int nr = *it;
    int in = g.nodes[nr].inputs[0];
    for (int v : g.nodes[in].vars) {
      if (contains(avail, v)) continue;
      ExP ne = view_expr(g, nr, v);
      std::unordered_map<int, int64_t> vs = {{v, g.var_sizes.at(v)}};
      for (auto& e : acc.idx)
        e = ex_simplify(ex_reify_sizes(ex_replace_var(e, v, ne), vs));
    }
  }
  for (auto& e : acc.idx) e = ex_simplify(ex_reify_sizes(e, g.var_sizes));
  return acc;
}

bool to_affine(const ExP& e, std::map<int, int64_t>& coef, int64_t& off,
               int64_t scale) {
  switch (e->op) {
    case EOp::value: off += scale * e->val; return true;
    case EOp::var: coef[e->var] += scale; return true;
    case EOp::add:
      return to_affine(e->a, coef, off, scale) &&
             to_affine(e->b, coef, off, scale);
    case EOp::negate: return to_affine(e->a, coef, off, -scale);
    case EOp::multiply: {
      int64_t c;
      if (ex_is_val(ex_simplify(e->a), &c))
        return to_affine(e->b, coef, off, scale * c);
      if (ex_is_val(ex_simplify(e->b), &c))
        return to_affine(e->a, coef, off, scale * c);
      return false;
    }
    default: return false;
  }
}

struct Builder {
  const IRGraph& g;
  const LowerOptions& opt;
  Plan plan;
  std::map<int, BufferInfo> bufs;  // node -> buffer holding its value
  std::vector<bool> mat;           // compute nodes materialised in HBM

  Builder(const IRGraph& g_, const LowerOptions& o) : g(g_), opt(o) {}

  int64_t vsize(int v) const { return g.var_sizes.at(v); }
  // position of var v's first loop in node N's order (after every loop
  // when N has no loop over v)
  static int order_pos(const Node& N, int v) {
    for (size_t i = 0; i < N.order.size(); ++i)
      if (N.order[i].first == v) return (int)i;
    return 1 << 20;
  }

  BufferInfo make_buf(int slot, const std::vector<int>& layout, bool scratch) {
    BufferInfo b;
    b.slot = slot;
    b.layout = layout;
    b.scratch = scratch;
    for (int v : layout) {
      b.sizes.push_back(vsize(v));
      b.elems *= vsize(v);
    }
    return b;
  }

  // ------------------------------------------------------- stage assembly
  struct StageCtx {
    PlanStage ps;
    std::vector<int> dims;  // stage vars
    int depth = 0, max_depth = 0;
  };

  int dim_of(const StageCtx& s, int var) const {
    auto it = std::find(s.dims.begin(), s.dims.end(), var);
    return it == s.dims.end() ? -1 : (int)(it - s.dims.begin());
  }

  void push_instr(StageCtx& s, uint8_t op, uint8_t arg, int delta) {
    auto& d = s.ps.dev;
    LTB_CHECK(d.ninstr < LTB_MAXI, "expression too large for one stage");
    d.code[d.ninstr++] = LtbVInstr{op, arg};
    s.depth += delta;
    s.max_depth = std::max(s.max_depth, s.depth);
    LTB_CHECK(s.max_depth <= LTB_STACK, "expression too deep for one stage");
  }

  void emit_qexpr(StageCtx& s, const ExP& e) {
    auto& d = s.ps.dev;
    auto word = [&](int32_t op, int32_t arg, int64_t imm) {
      LTB_CHECK(d.nq < LTB_MAXQ, "index program too long");
      d.q[d.nq++] = LtbQWord{op, arg, imm};
    };
    switch (e->op) {
      case EOp::value: word(LTB_Q_CONST, 0, e->val); return;
      case EOp::var: {
        int k = dim_of(s, e->var);
        if (k < 0) word(LTB_Q_CONST, 0, 0);  // out-of-scope var reads index 0
        else word(LTB_Q_COORD, k, 0);
        return;
      }
      case EOp::negate: emit_qexpr(s, e->a); word(LTB_Q_NEG, 0, 0); return;
      default: break;
    }
    LTB_CHECK(e->b, "unsupported index expression " << ex_str(e));
    emit_qexpr(s, e->a);
    emit_qexpr(s, e->b);
    switch (e->op) {
      case EOp::add: word(LTB_Q_ADD, 0, 0); return;
      case EOp::multiply: word(LTB_Q_MUL, 0, 0); return;
      case EOp::divide: word(LTB_Q_DIV, 0, 0); return;
      case EOp::modulo: word(LTB_Q_MOD, 0, 0); return;
      case EOp::max: word(LTB_Q_MAX, 0, 0); return;
      default: break;
    }
    throw Error("unsupported index expression " + ex_str(e));
  }

  // One leaf load of `buf` at per-layout-dim index expressions.
  int add_load(StageCtx& s, const BufferInfo& buf, std::vector<ExP> idx) {
    auto& d = s.ps.dev;
    // vars not iterated by this stage read index 0 (scoped exprs,
    // compile.cpp:858-872)
    std::unordered_map<int, int64_t> sz;
    for (int v : s.dims) sz[v] = vsize(v);
    for (auto& e : idx) {
      std::vector<int> vs;
      ex_vars(e, vs, false);
      for (int v : vs)
        if (dim_of(s, v) < 0) e = ex_simplify(ex_replace_var(e, v, ex_val(0)));
    }
    LtbLoad L{};
    L.buf = buf.slot;
    const int nd = (int)buf.layout.size();
    std::vector<int64_t> stride(nd, 1);
    for (int k = nd - 2; k >= 0; --k) stride[k] = stride[k + 1] * buf.sizes[k + 1];
    bool affine = true;
    std::vector<std::map<int, int64_t>> dc(nd);
    std::vector<int64_t> doff(nd, 0);
    for (int k = 0; k < nd && affine; ++k)
      affine = to_affine(idx[k], dc[k], doff[k], 1);
    // dedupe identical loads
    auto need_guard = [&](int k) {
      int64_t lo, hi;
      if (!ex_range(idx[k], sz, &lo, &hi)) return true;
      return lo < 0 || hi >= buf.sizes[k];
    };
    if (affine) {
      L.g0 = d.nguard;
      for (int k = 0; k < nd; ++k) {
        for (auto& p : dc[k]) L.coef[dim_of(s, p.first)] += p.second * stride[k];
        L.off += doff[k] * stride[k];
        if (need_guard(k)) {
          LTB_CHECK(d.nguard < LTB_MAXG, "too many bound guards in one stage");
          LtbGuard G{};
          for (auto& p : dc[k]) G.coef[dim_of(s, p.first)] += p.second;
          G.off = doff[k];
          G.ub = buf.sizes[k];
          d.guards[d.nguard++] = G;
          L.ng++;
        }
      }
    } else {
      L.q0 = d.nq;
      for (int k = 0; k < nd; ++k) {
        emit_qexpr(s, idx[k]);
        LTB_CHECK(d.nq < LTB_MAXQ, "index program too long");
        d.q[d.nq++] = LtbQWord{LTB_Q_DIM, need_guard(k) ? 1 : 0, buf.sizes[k]};
      }
      L.nq = d.nq - L.q0;
    }
    for (int i = 0; i < d.nload; ++i) {
      const auto& o = d.loads[i];
      if (o.buf == L.buf && o.nq == 0 && L.nq == 0 &&
          !memcmp(o.coef, L.coef, sizeof(L.coef)) && o.off == L.off &&
          o.ng == L.ng &&
          (L.ng == 0 || !memcmp(&d.guards[o.g0], &d.guards[L.g0],
                                sizeof(LtbGuard) * L.ng))) {
        d.nguard -= L.ng;
        return i;
      }
    }
    LTB_CHECK(d.nload < LTB_MAXL, "too many distinct loads in one stage");
    d.loads[d.nload] = L;
    return d.nload++;
  }

  std::vector<ExP> to_layout(const Access& acc, const BufferInfo& buf) {
    const auto& bv = g.nodes[acc.base].vars;
    std::vector<ExP> out;
    for (int v : buf.layout) {
      auto it = std::find(bv.begin(), bv.end(), v);
      LTB_CHECK(it != bv.end(), "buffer layout does not match node vars");
      out.push_back(acc.idx[it - bv.begin()]);
    }
    return out;
  }

  void emit_value(StageCtx& s, int consumer, int input) {
    Access acc = derive_access(g, consumer, input);
    auto bit = bufs.find(acc.base);
    if (bit != bufs.end()) {
      int li = add_load(s, bit->second, to_layout(acc, bit->second));
      push_instr(s, LTB_V_LOAD, (uint8_t)li, +1);
      return;
    }
    const Node& B = g.nodes[acc.base];
    LTB_CHECK(is_compute(B.op) && !acc.through_view,
              "node %" << acc.base << " (" << op_name(B.op)
                       << ") has no materialised buffer");
    emit_node_value(s, acc.base);
  }

  void emit_op(StageCtx& s, Op op) {
    switch (op) {
      case Op::add: push_instr(s, LTB_V_ADD, 0, -1); break;
      case Op::subtract: push_instr(s, LTB_V_SUB, 0, -1); break;
      case Op::multiply: push_instr(s, LTB_V_MUL, 0, -1); break;
      case Op::divide: push_instr(s, LTB_V_DIV, 0, -1); break;
      case Op::min: push_instr(s, LTB_V_MIN, 0, -1); break;
      case Op::max: push_instr(s, LTB_V_MAX, 0, -1); break;
      case Op::exp: push_instr(s, LTB_V_EXP, 0, 0); break;
      case Op::log: push_instr(s, LTB_V_LOG, 0, 0); break;
      case Op::sqrt: push_instr(s, LTB_V_SQRT, 0, 0); break;
      case Op::abs: push_instr(s, LTB_V_ABS, 0, 0); break;
      case Op::negate: push_instr(s, LTB_V_NEG, 0, 0); break;
      case Op::reciprocal: push_instr(s, LTB_V_RECIP, 0, 0); break;
      default: throw Error(std::string("unsupported op ") + op_name(op));
    }
  }

  // Value of an elementwise compute node at the stage's iteration point
  // (compile.cpp:974-1081 / cpp.cpp:172-270 for one output element).
  void emit_node_value(StageCtx& s, int n) {
    const Node& N = g.nodes[n];
    LTB_CHECK(!N.inputs.empty(), "compute node without inputs");
    if (is_unary(N.op)) {
      LTB_CHECK(N.inputs.size() == 1, "unary op with several inputs");
      emit_value(s, n, N.inputs[0]);
      emit_op(s, N.op);
      return;
    }
    emit_value(s, n, N.inputs[0]);
    if (N.op == Op::copy) return;
    for (size_t i = 1; i < N.inputs.size(); ++i) {
      emit_value(s, n, N.inputs[i]);
      emit_op(s, N.op);
    }
  }

  void set_dims(StageCtx& s, const std::vector<int>& out,
                const std::vector<int>& red) {
    s.dims = out;
    s.dims.insert(s.dims.end(), red.begin(), red.end());
    LTB_CHECK(s.dims.size() <= LTB_MAXD,
              "loop nest deeper than " << LTB_MAXD << " vars");
    auto& d = s.ps.dev;
    d.ndim = (int)s.dims.size();
    d.nout = (int)out.size();
    d.red_total = 1;
    for (int k = 0; k < d.ndim; ++k) {
      d.size[k] = vsize(s.dims[k]);
      if (k >= d.nout) d.red_total *= d.size[k];
    }
    s.ps.dim_vars = s.dims;
  }

  void set_output(StageCtx& s, const BufferInfo& out) {
    auto& d = s.ps.dev;
    d.out_buf = out.slot;
    int64_t st = 1;
    for (int k = (int)out.layout.size() - 1; k >= 0; --k) {
      int dk = dim_of(s, out.layout[k]);
      LTB_CHECK(dk >= 0 && dk < d.nout, "output var not iterated");
      d.out_coef[dk] = st;
      st *= out.sizes[k];
    }
  }

  static int red_code(Op op) {
    switch (op) {
      case Op::add: return LTB_R_ADD;
      case Op::multiply: return LTB_R_MUL;
      case Op::max: return LTB_R_MAX;
      case Op::min: return LTB_R_MIN;
      case Op::subtract: return LTB_R_SUB;
      case Op::divide: return LTB_R_DIV;
      default: return LTB_R_NONE;
    }
  }

  // reset values (compile.cpp:217-271): add/sub 0, mul/div 1, min +FLT_MAX,
  // max -FLT_MAX
  static float red_init(int r) {
    switch (r) {
      case LTB_R_MUL:
      case LTB_R_DIV: return 1.f;
      case LTB_R_MAX: return -FLT_MAX;
      case LTB_R_MIN: return FLT_MAX;
      default: return 0.f;
    }
  }

  // Load modes, the linear fast path and 32-bit division constants.
  static void finalize(LtbStage& d) {
    bool linear = d.ndim == d.nout && d.nout > 0;
    for (int i = 0; i < d.nload; ++i) {
      LtbLoad& L = d.loads[i];
      L.mode = LTB_L_GENERAL;
      if (L.nq || L.ng) {
        linear = false;
        continue;
      }
      bool same = true, zero = true;
      for (int k = 0; k < d.ndim; ++k) {
        same = same && L.coef[k] == (k < d.nout ? d.out_coef[k] : 0);
        zero = zero && L.coef[k] == 0;
      }
      if (zero) L.mode = LTB_L_SCALAR;
      else if (same && d.ndim == d.nout) L.mode = LTB_L_LINEAR;
      else linear = false;
    }
    d.linear = linear ? 1 : 0;
    const int64_t lim = int64_t(1) << 31;
    int64_t outs = 1;
    bool small = true;
    for (int k = 0; k < d.ndim; ++k) {
      int64_t n = d.size[k];
      small = small && n < lim;
      if (k < d.nout) outs *= n;
      uint32_t l = 0;
      while (l < 32 && (int64_t(1) << l) < n) ++l;
      uint64_t m = n < lim && n > 0
                       ? (((uint64_t(1) << 32) * ((uint64_t(1) << l) - n)) / n) + 1
                       : 1;
      d.dm_mul[k] = (uint32_t)m;
      d.dm_shr[k] = l;
    }
    d.small = small && outs < lim && d.red_total < lim;
  }

  // ------------------------------------------------------------- lowering
  void detect_contraction(StageCtx& s, int R) {
    const auto& d = s.ps.dev;
    if (d.red_op != LTB_R_ADD || d.nload != 2 || d.ninstr != 4) return;
    if (!(d.code[0].op == LTB_V_LOAD && d.code[1].op == LTB_V_LOAD &&
          d.code[2].op == LTB_V_MUL && d.code[3].op == LTB_V_FOLD))
      return;
    if (d.loads[0].nq || d.loads[1].nq) return;
    Contraction c;
    const LtbLoad& A = d.loads[d.code[0].arg];
    const LtbLoad& B = d.loads[d.code[1].arg];
    auto uses = [&](const LtbLoad& L, int k) {
      if (L.coef[k]) return true;
      for (int gi = L.g0; gi < L.g0 + L.ng; ++gi)
        if (d.guards[gi].coef[k]) return true;
      return false;
    };
    for (int k = 0; k < d.ndim; ++k) {
      bool ia = uses(A, k), ib = uses(B, k);
      int v = s.dims[k];
      if (k < d.nout) {
        if (ia && ib) c.bvars.push_back(v);
        else if (ia) c.mvars.push_back(v);
        else if (ib) c.nvars.push_back(v);
        else return;  // output var neither operand uses
      } else {
        if (!(ia && ib)) return;
        c.kvars.push_back(v);
      }
    }
    if (c.mvars.empty() || c.nvars.empty() || c.kvars.empty()) return;
    for (int v : c.bvars) c.B *= vsize(v);
    for (int v : c.mvars) c.M *= vsize(v);
    for (int v : c.nvars) c.N *= vsize(v);
    for (int v : c.kvars) c.K *= vsize(v);
    c.a_load = d.code[0].arg;
    c.b_load = d.code[1].arg;
    c.a_guarded = A.ng > 0;
    c.b_guarded = B.ng > 0;
    s.ps.con = c;
    s.ps.family = Family::contraction;
  }

  void choose_reduce_family(StageCtx& s) {
    auto& d = s.ps.dev;
    int64_t outs = 1;
    for (int k = 0; k < d.nout; ++k) outs *= d.size[k];
    const int64_t R = d.red_total;
    // the innermost reduced dim is contiguous in the first load?
    bool red_contig = d.nload > 0 && d.loads[0].nq == 0 &&
                      d.loads[0].coef[d.ndim - 1] == 1;
    bool parallel_ok = d.red_op == LTB_R_ADD || d.red_op == LTB_R_MUL ||
                       d.red_op == LTB_R_MAX || d.red_op == LTB_R_MIN;
    if (R <= 64 || !parallel_ok) {
      s.ps.family = Family::reduce_serial;
    } else if (!red_contig && outs >= 148 * 128) {
      s.ps.family = Family::reduce_serial;  // coalesced across outputs
    } else if (outs < 2 * 148 && R >= 65536 &&
               (d.red_op == LTB_R_ADD || d.red_op == LTB_R_MUL)) {
      s.ps.family = Family::reduce_split;
    } else {
      s.ps.family = Family::reduce_parallel;
    }
    if (d.red_op == LTB_R_ADD && R > opt.kahan_threshold) d.kahan = 1;
  }

  // Loop annotations of the stage's node N: backend sub-tree annotations
  // ("[cuda]": this backend; any other backend is rejected, there is no
  // host path to hand a sub-tree to) and the launch pins (StagePins).
  void read_pins(StageCtx& s, const Node& N) {
    StagePins& p = s.ps.pins;
    auto& d = s.ps.dev;
    std::ostringstream notes;
    std::vector<int64_t> par_out;  // iteration counts, outermost first
    for (size_t i = 0; i < N.order.size() && i < N.loop_annotations.size(); ++i) {
      const int v = N.order[i].first;
      const int64_t iters = N.order[i].second.size + (N.order[i].second.tail > 0 ? 1 : 0);
      const int k = dim_of(s, v);
      std::istringstream words(N.loop_annotations[i]);
      for (std::string w; words >> w;) {
        if (w.size() > 2 && w.front() == '[' && w.back() == ']') {
          const std::string be = w.substr(1, w.size() - 2);
          LTB_CHECK(be == "cuda", "loop " << g.var_names[v] << " is annotated for backend '" << be
                                          << "': this backend runs every loop on the device "
                                             "and has no other backend to hand a sub-tree to");
          notes << " [cuda] sub-tree at loop " << g.var_names[v]
                << ": device launches with the rest of the tree, the loops around it in the "
                   "grid (no host loop);";
        } else if (w == "parallel") {
          if (k >= 0 && k < d.nout) par_out.push_back(iters);
          else if (k >= d.nout) p.parallel_red = (p.parallel_red ? p.parallel_red : 1) * iters;
        } else if (w == "unroll") {
          p.unroll = (int)std::min<int64_t>(iters, 1 << 20);
        } else if (w == "vectorize") {
          notes << " vectorize at " << g.var_names[v]
                << ": 16-byte vectors are used wherever alignment allows (no change);";
        } else {
          notes << " annotation '" << w << "' at " << g.var_names[v] << " ignored;";
        }
      }
    }
    if (!par_out.empty()) {
      p.parallel_out = 1;
      for (auto x : par_out) p.parallel_out *= x;
      if (par_out.size() >= 2) p.cta_threads = (int)std::min<int64_t>(par_out.back(), 1 << 20);
    }
    // a parallel loop over a reduced var asks for a parallel reduction: a
    // tree per output up to 256 threads, split-K partials beyond that
    const bool tree_ok = d.red_op == LTB_R_ADD || d.red_op == LTB_R_MUL ||
                         d.red_op == LTB_R_MAX || d.red_op == LTB_R_MIN;
    if (p.parallel_red > 1 && tree_ok && s.ps.family == Family::reduce_serial)
      s.ps.family = Family::reduce_parallel;
    if (p.parallel_red > 256 && s.ps.family == Family::reduce_parallel &&
        (d.red_op == LTB_R_ADD || d.red_op == LTB_R_MUL))
      s.ps.family = Family::reduce_split;
    // Sums: a sequential fold (reduce_serial) is the reference's own
    // order, bit for bit; a tree or split-K sum reassociates, so it is
    // compensated (TwoSum partials, error ~2u|sum|): plain trees have errors
    // of the reference's size in other places, which entry by entry exceed
    // the reference's on some cancelling sums.
    if (d.red_op == LTB_R_ADD &&
        (s.ps.family == Family::reduce_parallel || s.ps.family == Family::reduce_split))
      d.kahan = 1;
    if (s.ps.family == Family::contraction && p.any()) {
      notes << " parallel/unroll on a contraction: the tile kernel keeps its own mapping;";
      p.parallel_out = p.parallel_red = 0;
      p.cta_threads = p.unroll = 0;
    }
    p.text = notes.str();
  }

  std::string stage_text(const StageCtx& s) {
    std::ostringstream ss;
    const auto& d = s.ps.dev;
    ss << family_name(s.ps.family) << " %" << s.ps.node << " [";
    for (int k = 0; k < d.ndim; ++k) {
      if (k == d.nout) ss << " | ";
      else if (k) ss << ", ";
      ss << g.var_names[s.dims[k]] << ":" << d.size[k];
    }
    ss << "] -> buf" << d.out_buf << " loads=" << d.nload
       << " guards=" << d.nguard << " instrs=" << d.ninstr;
    if (d.red_op) ss << " red=" << d.red_op << (d.kahan ? "(kahan)" : "");
    if (s.ps.family == Family::contraction) {
      const auto& c = s.ps.con;
      ss << " gemm B=" << c.B << " M=" << c.M << " N=" << c.N << " K=" << c.K
         << (c.a_guarded ? " A-guarded" : "");
    }
    const StagePins& p = s.ps.pins;
    if (p.any()) {
      ss << " pinned{";
      if (p.parallel_out) ss << " parallel=" << p.parallel_out;
      if (p.cta_threads) ss << " cta=" << p.cta_threads;
      if (p.parallel_red) ss << " parallel_reduce=" << p.parallel_red;
      if (p.unroll) ss << " unroll=" << p.unroll;
      ss << " }";
    }
    if (!p.text.empty()) ss << " annotations:" << p.text;
    return ss.str();
  }

  void run() {
    const int nn = (int)g.nodes.size();
    plan.n_in = (int)g.inputs.size();
    plan.n_out = (int)g.outputs.size();
    for (int i = 0; i < plan.n_in; ++i) {
      int n = g.inputs[i];
      bufs[n] = make_buf(i, g.nodes[n].vars, false);
      plan.io_elems.push_back(bufs[n].elems);
    }
    for (int j = 0; j < plan.n_out; ++j) {
      int n = g.outputs[j];
      auto b = make_buf(plan.n_in + j, g.nodes[n].vars, false);
      plan.io_elems.push_back(b.elems);
      bufs[n] = b;
    }
    mat.assign(nn, false);
    for (int n = 0; n < nn; ++n) {
      const Node& N = g.nodes[n];
      if (is_compute(N.op) && !g.reduction_vars(n).empty()) {
        LTB_CHECK(!is_unary(N.op),
                  "unary op " << op_name(N.op) << " with reduced vars");
        LTB_CHECK(N.op != Op::copy, "copy with reduced vars");
        mat[n] = true;
      }
      if (N.op == Op::view || N.op == Op::read) continue;
      for (int x : N.inputs) {
        if (g.nodes[x].op != Op::view) continue;
        int b = x;
        while (g.nodes[b].op == Op::view) b = g.nodes[b].inputs[0];
        if (is_compute(g.nodes[b].op)) mat[b] = true;
      }
    }
    // writes whose input is a compute node write its value in place
    std::map<int, int> fused_write;  // compute node -> write node
    for (int w : g.outputs) {
      int y = g.nodes[w].inputs.at(0);
      const auto& wv = g.nodes[w].vars;
      const auto& yv = g.nodes[y].vars;
      bool perm = wv.size() == yv.size() &&
                  std::is_permutation(wv.begin(), wv.end(), yv.begin());
      if (is_compute(g.nodes[y].op) && perm && !fused_write.count(y))
        fused_write[y] = w;
    }
    for (int n = 0; n < nn; ++n) {
      if (!mat[n]) continue;
      if (fused_write.count(n)) {
        BufferInfo b = bufs.at(fused_write[n]);
        bufs[n] = b;
      } else {
        int slot = plan.num_slots();
        bufs[n] = make_buf(slot, g.nodes[n].vars, true);
        plan.scratch_elems.push_back(bufs[n].elems);
      }
    }
    for (int n : topo_order(g)) {
      const Node& N = g.nodes[n];
      bool is_write = N.op == Op::write;
      bool fused_elem = is_compute(N.op) && !mat[n] && fused_write.count(n);
      if (!(is_write || mat[n] || fused_elem)) continue;
      if (is_write) {
        int y = N.inputs.at(0);
        if (fused_write.count(y) && fused_write[y] == n) continue;
      }
      StageCtx s;
      s.ps.node = n;
      auto& d = s.ps.dev;
      if (is_write) {
        set_dims(s, N.vars, {});
        set_output(s, bufs.at(n));
        emit_value(s, n, N.inputs.at(0));
        s.ps.family = Family::elementwise;
      } else {
        const BufferInfo& out = fused_elem ? bufs.at(fused_write[n]) : bufs.at(n);
        // reduced vars in loop order (first appearance in the node's
        // order): the reference folds them in its loop nest's order
        // (compile.cpp:217-271 resets at the loops' LCA, then visits the
        // reduced points lexicographically in that order)
        auto red = g.reduction_vars(n);
        std::stable_sort(red.begin(), red.end(), [&](int a, int b) {
          return order_pos(N, a) < order_pos(N, b);
        });
        set_dims(s, out.layout, red);
        set_output(s, out);
        if (!red.empty()) {
          d.red_op = red_code(N.op);
          LTB_CHECK(d.red_op != LTB_R_NONE,
                    "cannot reduce with op " << op_name(N.op));
          d.red_init = red_init(d.red_op);
          for (int x : N.inputs) {
            emit_value(s, n, x);
            push_instr(s, LTB_V_FOLD, 0, -1);
          }
          detect_contraction(s, n);
          if (s.ps.family != Family::contraction) choose_reduce_family(s);
        } else {
          emit_node_value(s, n);
          s.ps.family = Family::elementwise;
        }
      }
      read_pins(s, N);
      finalize(s.ps.dev);
      s.ps.text = stage_text(s);
      plan.stages.push_back(s.ps);
    }
    if (opt.fuse_rows) group_rows();
    // compulsory traffic: every input read once, every output written once
    for (auto e : plan.io_elems) plan.algorithmic_bytes += 4 * e;
    for (auto& st : plan.stages)
      if (st.family == Family::contraction)
        plan.flops += 2.0 * st.con.B * st.con.M * st.con.N * st.con.K;
    std::ostringstream ss;
    ss << "[cuda sm_100a plan] " << plan.stages.size() << " stage(s), "
       << plan.scratch_elems.size() << " scratch buffer(s)\n";
    for (size_t i = 0; i < plan.stages.size(); ++i)
      ss << "  " << i << ": " << plan.stages[i].text << "\n";
    for (auto& grp : plan.row_groups) {
      ss << "  row_chain {";
      for (int i : grp) ss << " " << i;
      ss << " }\n";
    }
    plan.dump = ss.str();
  }

  // m = max_n x; s = sum_n exp(x - m); y = exp(x - m) / s over the same x
  // row with a unit inner stride: the fused row-softmax pattern.
  bool is_softmax(const std::vector<int>& grp) const {
    if (grp.size() != 3) return false;
    const auto& a = plan.stages[grp[0]].dev;
    const auto& b = plan.stages[grp[1]].dev;
    const auto& c = plan.stages[grp[2]].dev;
    auto ops = [](const LtbStage& d, std::vector<int> want) {
      if (d.ninstr != (int)want.size()) return false;
      for (int i = 0; i < d.ninstr; ++i)
        if (d.code[i].op != want[i]) return false;
      return true;
    };
    if (a.red_op != LTB_R_MAX || b.red_op != LTB_R_ADD) return false;
    if (!ops(a, {LTB_V_LOAD, LTB_V_FOLD})) return false;
    if (!ops(b, {LTB_V_LOAD, LTB_V_LOAD, LTB_V_SUB, LTB_V_EXP, LTB_V_FOLD})) return false;
    if (!ops(c, {LTB_V_LOAD, LTB_V_LOAD, LTB_V_SUB, LTB_V_EXP, LTB_V_LOAD, LTB_V_DIV}))
      return false;
    auto same_x = [](const LtbStage& p, int pi, const LtbStage& q, int qi) {
      const LtbLoad& x = p.loads[p.code[pi].arg];
      const LtbLoad& y = q.loads[q.code[qi].arg];
      if (x.buf != y.buf || x.off != y.off || x.nq || y.nq || x.ng || y.ng) return false;
      for (int k = 0; k < p.ndim; ++k)
        if (x.coef[k] != y.coef[k]) return false;
      return true;
    };
    // x loads agree (row dims then the inner dim, same positions in all
    // three stages by construction of the group)
    if (!same_x(a, 0, b, 0) || !same_x(a, 0, c, 0)) return false;
    const LtbLoad& x = a.loads[a.code[0].arg];
    if (x.coef[a.ndim - 1] != 1) return false;
    // m and s are the first two stages' per-row outputs
    if (b.loads[b.code[1].arg].buf != a.out_buf) return false;
    if (c.loads[c.code[1].arg].buf != a.out_buf) return false;
    if (c.loads[c.code[4].arg].buf != b.out_buf) return false;
    if (c.out_coef[c.nout - 1] != 1) return false;
    return true;
  }

  // Consecutive stages that iterate the same outer "row" vars and only
  // exchange per-row scalars fuse into one row_chain launch (row softmax,
  // normalisation chains): one CTA owns a row for the whole chain.
  void group_rows() {
    auto& st = plan.stages;
    size_t i = 0;
    while (i < st.size()) {
      auto row_of = [&](const PlanStage& p, std::vector<int>& rows,
                        std::vector<int>& inner) -> bool {
        const auto& d = p.dev;
        if (p.family == Family::contraction) return false;
        if (p.family == Family::elementwise) {
          if (d.nout < 2) return false;
          rows.assign(p.dim_vars.begin(), p.dim_vars.begin() + d.nout - 1);
          inner.assign(p.dim_vars.begin() + d.nout - 1, p.dim_vars.end());
          return true;
        }
        if (d.red_op != LTB_R_ADD && d.red_op != LTB_R_MAX &&
            d.red_op != LTB_R_MIN && d.red_op != LTB_R_MUL)
          return false;
        rows.assign(p.dim_vars.begin(), p.dim_vars.begin() + d.nout);
        inner.assign(p.dim_vars.begin() + d.nout, p.dim_vars.end());
        return true;
      };
      std::vector<int> rows0, inner0;
      if (!row_of(st[i], rows0, inner0) || st[i].family == Family::elementwise ||
          inner0.size() != 1) {
        ++i;
        continue;
      }
      int64_t inner_n = vsize(inner0[0]);
      std::vector<int> grp = {(int)i};
      std::set<int> row_scalars = {st[i].dev.out_buf};
      size_t j = i + 1;
      for (; j < st.size(); ++j) {
        std::vector<int> r, in;
        if (!row_of(st[j], r, in)) break;
        if (r != rows0 || in != inner0) break;
        grp.push_back((int)j);
        if (st[j].family != Family::elementwise) row_scalars.insert(st[j].dev.out_buf);
        else { ++j; break; }  // chain ends at its per-element output
      }
      bool ends_elem = st[grp.back()].family == Family::elementwise;
      if (grp.size() >= 2 && ends_elem && inner_n <= 16384 && inner_n >= 256) {
        plan.row_groups.push_back(grp);
        for (int k : grp) {
          st[k].family = Family::row_chain;
          // fused row chains compensate only long rows
          if (st[k].dev.red_op == LTB_R_ADD && st[k].dev.red_total <= opt.kahan_threshold &&
              st[k].dev.kahan) {
            st[k].dev.kahan = 0;
            const size_t at = st[k].text.find("(kahan)");
            if (at != std::string::npos) st[k].text.erase(at, 7);
          }
          if (st[k].pins.any()) {  // the fused row kernel has its own mapping
            st[k].pins = StagePins{};
            st[k].text += " (parallel/unroll not applied: fused into a row chain)";
          }
        }
        for (size_t k = 0; k < grp.size(); ++k) st[grp[k]].rows_from = grp[0];
        if (is_softmax(grp))
          for (int k : grp) st[k].dev.pattern = LTB_P_SOFTMAX;
        i = j;
      } else {
        ++i;
      }
    }
  }
};

}  // namespace

Plan lower(const IRGraph& g, const LowerOptions& opt) {
  Builder b(g, opt);
  b.run();
  return std::move(b.plan);
}

}  // namespace ltb
