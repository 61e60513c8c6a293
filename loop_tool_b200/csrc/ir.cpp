#include "ir.hpp"

#include <algorithm>
#include <cmath>
#include <functional>
#include <limits>
#include <set>
#include <sstream>

namespace ltb {

const char* op_name(Op op) {
  switch (op) {
    case Op::constant: return "constant";
    case Op::write: return "write";
    case Op::read: return "read";
    case Op::view: return "view";
    case Op::copy: return "copy";
    case Op::add: return "add";
    case Op::subtract: return "subtract";
    case Op::multiply: return "multiply";
    case Op::divide: return "divide";
    case Op::min: return "min";
    case Op::max: return "max";
    case Op::log: return "log";
    case Op::exp: return "exp";
    case Op::sqrt: return "sqrt";
    case Op::abs: return "abs";
    case Op::negate: return "negate";
    case Op::reciprocal: return "reciprocal";
    case Op::name: return "name";
  }
  return "?";
}

// ------------------------------------------------------------ expressions
ExP ex_val(int64_t v) {
  auto e = std::make_shared<Ex>();
  e->op = EOp::value;
  e->val = v;
  return e;
}
ExP ex_var(int v) {
  auto e = std::make_shared<Ex>();
  e->op = EOp::var;
  e->var = v;
  return e;
}
ExP ex_size(int v) {
  auto e = std::make_shared<Ex>();
  e->op = EOp::size;
  e->var = v;
  return e;
}
ExP ex_un(EOp op, ExP a) {
  auto e = std::make_shared<Ex>();
  e->op = op;
  e->a = std::move(a);
  return e;
}
ExP ex_bin(EOp op, ExP a, ExP b) {
  auto e = std::make_shared<Ex>();
  e->op = op;
  e->a = std::move(a);
  e->b = std::move(b);
  return e;
}

bool ex_is_val(const ExP& e, int64_t* v) {
  if (e->op != EOp::value) return false;
  if (v) *v = e->val;
  return true;
}

bool ex_equal(const ExP& x, const ExP& y) {
  if (x.get() == y.get()) return true;
  if (x->op != y->op) return false;
  switch (x->op) {
    case EOp::value: return x->val == y->val;
    case EOp::var:
    case EOp::size: return x->var == y->var;
    default: break;
  }
  if (!!x->a != !!y->a || !!x->b != !!y->b) return false;
  if (x->a && !ex_equal(x->a, y->a)) return false;
  if (x->b && !ex_equal(x->b, y->b)) return false;
  return true;
}

void ex_vars(const ExP& e, std::vector<int>& out, bool include_sized) {
  if (e->op == EOp::var || (include_sized && e->op == EOp::size)) {
    if (std::find(out.begin(), out.end(), e->var) == out.end())
      out.push_back(e->var);
    return;
  }
  if (e->a) ex_vars(e->a, out, include_sized);
  if (e->b) ex_vars(e->b, out, include_sized);
}

bool ex_contains(const ExP& e, int var) {
  if (e->op == EOp::var || e->op == EOp::size) return e->var == var;
  return (e->a && ex_contains(e->a, var)) || (e->b && ex_contains(e->b, var));
}

ExP ex_replace_var(const ExP& e, int var, const ExP& with) {
  if (e->op == EOp::var) return e->var == var ? with : e;
  if (e->op == EOp::value || e->op == EOp::size) return e;
  auto a = e->a ? ex_replace_var(e->a, var, with) : nullptr;
  auto b = e->b ? ex_replace_var(e->b, var, with) : nullptr;
  if (a.get() == e->a.get() && b.get() == e->b.get()) return e;
  return b ? ex_bin(e->op, a, b) : ex_un(e->op, a);
}

ExP ex_reify_sizes(const ExP& e,
                   const std::unordered_map<int, int64_t>& sz) {
  if (e->op == EOp::size) {
    auto it = sz.find(e->var);
    return it == sz.end() ? e : ex_val(it->second);
  }
  if (e->op == EOp::value || e->op == EOp::var) return e;
  auto a = e->a ? ex_reify_sizes(e->a, sz) : nullptr;
  auto b = e->b ? ex_reify_sizes(e->b, sz) : nullptr;
  if (a.get() == e->a.get() && b.get() == e->b.get()) return e;
  return b ? ex_bin(e->op, a, b) : ex_un(e->op, a);
}

// C semantics for int64 / and % (truncation toward zero).
static int64_t cdiv(int64_t a, int64_t b) { return a / b; }
static int64_t cmod(int64_t a, int64_t b) { return a % b; }

ExP ex_simplify(const ExP& e) {
  if (e->op == EOp::value || e->op == EOp::var || e->op == EOp::size)
    return e;
  ExP a = e->a ? ex_simplify(e->a) : nullptr;
  ExP b = e->b ? ex_simplify(e->b) : nullptr;
  int64_t va = 0, vb = 0;
  bool ca = a && ex_is_val(a, &va), cb = b && ex_is_val(b, &vb);
  switch (e->op) {
    case EOp::add:
      if (ca && cb) return ex_val(va + vb);
      if (ca && va == 0) return b;
      if (cb && vb == 0) return a;
      // fold constants through nested sums: c1 + (c2 + x)
      if (ca && b->op == EOp::add && ex_is_val(b->a))
        return ex_simplify(ex_bin(EOp::add, ex_val(va + b->a->val), b->b));
      if (cb && a->op == EOp::add && ex_is_val(a->b))
        return ex_simplify(ex_bin(EOp::add, a->a, ex_val(vb + a->b->val)));
      break;
    case EOp::multiply:
      if (ca && cb) return ex_val(va * vb);
      if ((ca && va == 0) || (cb && vb == 0)) return ex_val(0);
      if (ca && va == 1) return b;
      if (cb && vb == 1) return a;
      break;
    case EOp::divide:
      if (ca && cb && vb != 0 && va % vb == 0) return ex_val(va / vb);
      if (cb && vb == 1) return a;
      break;
    case EOp::modulo:
      if (ca && cb && vb != 0) return ex_val(cmod(va, vb));
      if (cb && vb == 1) return ex_val(0);
      break;
    case EOp::max:
      if (ca && cb) return ex_val(std::max(va, vb));
      if (ex_equal(a, b)) return a;
      break;
    case EOp::negate:
      if (ca) return ex_val(-va);
      if (a->op == EOp::negate) return a->a;
      break;
    default:
      break;
  }
  if (a.get() == e->a.get() && b.get() == e->b.get()) return e;
  return b ? ex_bin(e->op, a, b) : ex_un(e->op, a);
}

ExP ex_diff(const ExP& e, int var) {
  if (!ex_contains(e, var)) return ex_val(0);
  if (e->op == EOp::var) return ex_val(1);
  if (e->op == EOp::size) return ex_val(0);  // |v| does not vary with v
  const ExP& a = e->a;
  const ExP& b = e->b;
  switch (e->op) {
    case EOp::add: {
      bool ia = ex_contains(a, var), ib = ex_contains(b, var);
      if (ia && !ib) return ex_diff(a, var);
      if (ib && !ia) return ex_diff(b, var);
      return ex_bin(EOp::add, ex_diff(a, var), ex_diff(b, var));
    }
    case EOp::multiply: {
      bool ia = ex_contains(a, var), ib = ex_contains(b, var);
      if (ia && !ib) return ex_bin(EOp::multiply, ex_diff(a, var), b);
      if (ib && !ia) return ex_bin(EOp::multiply, ex_diff(b, var), a);
      return ex_bin(EOp::add, ex_bin(EOp::multiply, ex_diff(a, var), b),
                    ex_bin(EOp::multiply, ex_diff(b, var), a));
    }
    case EOp::divide: {
      bool ia = ex_contains(a, var), ib = ex_contains(b, var);
      if (ia && !ib) return ex_bin(EOp::divide, ex_diff(a, var), b);
      auto bb = ex_bin(EOp::multiply, b, b);
      if (ib && !ia)
        return ex_bin(EOp::divide, ex_bin(EOp::multiply, a, ex_diff(b, var)),
                      bb);
      return ex_bin(
          EOp::divide,
          ex_bin(EOp::add, ex_bin(EOp::multiply, ex_diff(a, var), b),
                 ex_un(EOp::negate, ex_bin(EOp::multiply, a, ex_diff(b, var)))),
          bb);
    }
    case EOp::negate:
      return ex_un(EOp::negate, ex_diff(a, var));
    case EOp::reciprocal:
      return ex_bin(EOp::divide, ex_diff(a, var), ex_bin(EOp::multiply, a, a));
    default:
      break;
  }
  throw Error("cannot differentiate expression " + ex_str(e));
}

bool ex_eval(const ExP& e, const std::unordered_map<int, int64_t>& env,
             int64_t* out) {
  switch (e->op) {
    case EOp::value: *out = e->val; return true;
    case EOp::var:
    case EOp::size: {
      auto it = env.find(e->var);
      if (it == env.end()) return false;
      *out = it->second;
      return true;
    }
    default: break;
  }
  int64_t x = 0, y = 0;
  if (!ex_eval(e->a, env, &x)) return false;
  if (e->b && !ex_eval(e->b, env, &y)) return false;
  switch (e->op) {
    case EOp::add: *out = x + y; return true;
    case EOp::multiply: *out = x * y; return true;
    case EOp::divide:
      if (y == 0) return false;
      *out = cdiv(x, y);
      return true;
    case EOp::modulo:
      if (y == 0) return false;
      *out = cmod(x, y);
      return true;
    case EOp::max: *out = std::max(x, y); return true;
    case EOp::negate: *out = -x; return true;
    case EOp::reciprocal:
      if (x == 0) return false;
      *out = cdiv(1, x);
      return true;
    default: return false;
  }
}

bool ex_eval_float(const ExP& e, float* out) {
  switch (e->op) {
    case EOp::value: *out = (float)e->val; return true;
    case EOp::var:
    case EOp::size: return false;
    default: break;
  }
  float x = 0, y = 0;
  if (!ex_eval_float(e->a, &x)) return false;
  if (e->b && !ex_eval_float(e->b, &y)) return false;
  switch (e->op) {
    case EOp::add: *out = x + y; return true;
    case EOp::multiply: *out = x * y; return true;
    case EOp::divide: *out = x / y; return true;
    case EOp::modulo: *out = (float)((int64_t)x % (int64_t)y); return true;
    case EOp::max: *out = std::max(x, y); return true;
    case EOp::negate: *out = -x; return true;
    default: return false;
  }
}

bool ex_range(const ExP& e, const std::unordered_map<int, int64_t>& sz,
              int64_t* lo, int64_t* hi) {
  switch (e->op) {
    case EOp::value: *lo = *hi = e->val; return true;
    case EOp::var: {
      auto it = sz.find(e->var);
      if (it == sz.end()) return false;
      *lo = 0;
      *hi = std::max<int64_t>(it->second - 1, 0);
      return true;
    }
    case EOp::size: {
      auto it = sz.find(e->var);
      if (it == sz.end()) return false;
      *lo = *hi = it->second;
      return true;
    }
    default: break;
  }
  int64_t al, ah, bl = 0, bh = 0;
  if (!ex_range(e->a, sz, &al, &ah)) return false;
  if (e->b && !ex_range(e->b, sz, &bl, &bh)) return false;
  switch (e->op) {
    case EOp::add: *lo = al + bl; *hi = ah + bh; return true;
    case EOp::negate: *lo = -ah; *hi = -al; return true;
    case EOp::multiply: {
      int64_t c[4] = {al * bl, al * bh, ah * bl, ah * bh};
      *lo = *std::min_element(c, c + 4);
      *hi = *std::max_element(c, c + 4);
      return true;
    }
    case EOp::divide:
      if (bl != bh || bl <= 0) return false;  // only positive constants
      *lo = cdiv(al, bl);
      *hi = cdiv(ah, bl);
      return true;
    case EOp::modulo:
      if (bl != bh || bl <= 0) return false;
      if (al >= 0 && ah < bl) {
        *lo = al;
        *hi = ah;
      } else if (al >= 0) {
        *lo = 0;
        *hi = bl - 1;
      } else {
        *lo = -(bl - 1);
        *hi = bl - 1;
      }
      return true;
    case EOp::max:
      *lo = std::max(al, bl);
      *hi = std::max(ah, bh);
      return true;
    default: return false;
  }
}

std::string ex_str(const ExP& e, const std::vector<std::string>* names) {
  std::ostringstream ss;
  switch (e->op) {
    case EOp::value: ss << e->val; break;
    case EOp::var:
      if (names && e->var >= 0 && e->var < (int)names->size())
        ss << (*names)[e->var];
      else
        ss << "v" << e->var;
      break;
    case EOp::size:
      ss << "|" << (names && e->var < (int)names->size() ? (*names)[e->var]
                                                          : "v" + std::to_string(e->var))
         << "|";
      break;
    case EOp::negate: ss << "-(" << ex_str(e->a, names) << ")"; break;
    case EOp::reciprocal: ss << "(1/" << ex_str(e->a, names) << ")"; break;
    case EOp::max:
      ss << "max(" << ex_str(e->a, names) << ", " << ex_str(e->b, names) << ")";
      break;
    default: {
      const char* o = e->op == EOp::add ? "+"
                      : e->op == EOp::multiply ? "*"
                      : e->op == EOp::divide ? "/"
                                             : "%";
      ss << "(" << ex_str(e->a, names) << o << ex_str(e->b, names) << ")";
    }
  }
  return ss.str();
}

// ---------------------------------------------------------------- parsing
static std::vector<std::string> split(const std::string& s, char d) {
  // std::getline semantics, as the reference parser uses: a trailing
  // delimiter does not produce a final empty field.
  std::vector<std::string> out;
  std::istringstream ss(s);
  for (std::string t; std::getline(ss, t, d);) out.push_back(t);
  return out;
}

static int64_t to_i64(const std::string& s) {
  LTB_CHECK(!s.empty(), "empty integer field in IR text");
  size_t pos = 0;
  int64_t v = std::stoll(s, &pos);
  LTB_CHECK(pos == s.size(), "bad integer '" << s << "' in IR text");
  return v;
}

// Expression leaves hold the symbol's first-occurrence index until the
// node's sym->var map is known; remapped afterwards.
static ExP parse_expr(const std::string& str, std::set<int>& sym_idx,
                      int32_t& idx) {
  LTB_CHECK(!str.empty(), "empty expression in IR text");
  std::unordered_map<int32_t, ExP> idx_map;
  for (const auto& tok : split(str, ';')) {
    auto f = split(tok, '|');
    LTB_CHECK(f.size() == 3 || (f.size() == 2 && f[1] == "f"),
              "bad expression token '" << tok << "'");
    int32_t op = (int32_t)to_i64(f[0]);
    const std::string& ty = f[1];
    if (ty == "s") {
      sym_idx.insert(idx);
      idx_map[idx] = ex_var(idx);  // placeholder: var id == symbol index
    } else if (ty == "r") {
      int32_t ref = (int32_t)to_i64(f[2]);
      LTB_CHECK(sym_idx.count(ref), "dangling symbol reference " << ref);
      sym_idx.insert(idx);
      // an 'r' token aliases the symbol first seen at index ref
      idx_map[idx] = ex_var(ref);
    } else if (ty == "v") {
      idx_map[idx] = ex_val(to_i64(f[2]));
    } else if (ty == "f") {
      std::vector<ExP> args;
      for (const auto& a : split(f.size() > 2 ? f[2] : "", ',')) {
        int32_t ai = (int32_t)to_i64(a);
        auto it = idx_map.find(ai);
        if (sym_idx.count(ai) && it == idx_map.end()) {
          args.push_back(ex_var(ai));
        } else {
          LTB_CHECK(it != idx_map.end(), "unknown expression index " << ai);
          args.push_back(it->second);
        }
      }
      EOp eop = static_cast<EOp>(op);
      if (args.size() == 2) {
        LTB_CHECK(op >= 4 && op <= 8, "bad binary expression op " << op);
        idx_map[idx] = ex_bin(eop, args[0], args[1]);
      } else if (args.size() == 1) {
        LTB_CHECK(op >= 1 && op <= 3, "bad unary expression op " << op);
        if (eop == EOp::size) {
          LTB_CHECK(args[0]->op == EOp::var, "size() of a non-symbol");
          idx_map[idx] = ex_size(args[0]->var);
        } else {
          idx_map[idx] = ex_un(eop, args[0]);
        }
      } else {
        throw Error("cannot parse an empty function call in IR text");
      }
    } else {
      throw Error("invalid expression token type '" + ty + "'");
    }
    idx++;
  }
  return idx_map.at(idx - 1);
}

static ExP remap_syms(const ExP& e, const std::unordered_map<int, int>& m) {
  if (e->op == EOp::var || e->op == EOp::size) {
    auto it = m.find(e->var);
    LTB_CHECK(it != m.end(), "constraint symbol #" << e->var
                                                   << " is not mapped to a variable");
    return e->op == EOp::var ? ex_var(it->second) : ex_size(it->second);
  }
  if (e->op == EOp::value) return e;
  auto a = remap_syms(e->a, m);
  auto b = e->b ? remap_syms(e->b, m) : nullptr;
  return b ? ex_bin(e->op, a, b) : ex_un(e->op, a);
}

IRGraph parse_ir(const std::string& text) {
  IRGraph g;
  std::istringstream ss(text);
  for (std::string line; std::getline(ss, line);) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    if (line.empty()) continue;
    auto ch = split(line, ':');
    LTB_CHECK(!ch.empty(), "empty IR line");
    if (ch[0] == "v") {
      LTB_CHECK(ch.size() == 2, "invalid var line: " << line);
      g.var_names.push_back(ch[1]);
    } else if (ch[0] == "n") {
      // op:inputs:vars:constraints:symmap:priority:order:reuse:annots:annot
      while (ch.size() < 11) ch.push_back("");
      LTB_CHECK(ch.size() == 11, "invalid node line (" << ch.size()
                                                       << " fields): " << line);
      Node n;
      int32_t opc = (int32_t)to_i64(ch[1]);
      LTB_CHECK(opc >= 0 && opc <= 17, "unknown op code " << opc);
      n.op = static_cast<Op>(opc);
      for (auto& s : split(ch[2], ',')) n.inputs.push_back((int)to_i64(s));
      for (auto& s : split(ch[3], ',')) n.vars.push_back((int)to_i64(s));
      std::set<int> sym_idx;
      int32_t idx = 0;
      std::vector<std::pair<ExP, ExP>> raw;
      for (auto& cs : split(ch[4], '/')) {
        auto pos = cs.find('=');
        LTB_CHECK(pos != std::string::npos, "constraint without '='");
        auto l = parse_expr(cs.substr(0, pos), sym_idx, idx);
        auto r = parse_expr(cs.substr(pos + 1), sym_idx, idx);
        raw.emplace_back(l, r);
      }
      std::unordered_map<int, int> sym_to_var;
      for (auto& kv : split(ch[5], ',')) {
        auto pos = kv.find('=');
        LTB_CHECK(pos != std::string::npos, "bad sym map entry " << kv);
        sym_to_var[(int)to_i64(kv.substr(0, pos))] =
            (int)to_i64(kv.substr(pos + 1));
      }
      for (auto& p : raw)
        n.constraints.push_back({remap_syms(p.first, sym_to_var),
                                 remap_syms(p.second, sym_to_var)});
      n.priority = ch[6].empty() ? 0.f : std::stof(ch[6]);
      for (auto& o : split(ch[7], ',')) {
        auto t = split(o, ';');
        LTB_CHECK(t.size() == 3, "invalid order entry '" << o << "'");
        n.order.push_back({(int)to_i64(t[0]), {to_i64(t[1]), to_i64(t[2])}});
      }
      for (auto& s : split(ch[8], ',')) n.reuse_disabled.push_back((int)to_i64(s));
      n.loop_annotations = split(ch[9], ',');
      n.annotation = ch[10];
      if (n.op != Op::view)
        LTB_CHECK(n.constraints.empty(),
                  "constraints are only valid on view nodes");
      g.nodes.push_back(std::move(n));
    } else if (ch[0] == "i") {
      if (ch.size() > 1)
        for (auto& s : split(ch[1], ',')) g.inputs.push_back((int)to_i64(s));
    } else if (ch[0] == "o") {
      if (ch.size() > 1)
        for (auto& s : split(ch[1], ',')) g.outputs.push_back((int)to_i64(s));
    } else {
      throw Error("unknown IR line kind '" + ch[0] + "'");
    }
  }
  const int nn = (int)g.nodes.size(), nv = (int)g.var_names.size();
  LTB_CHECK(nn > 0, "IR has no nodes");
  for (int i = 0; i < nn; ++i) {
    auto& n = g.nodes[i];
    for (int inp : n.inputs) {
      LTB_CHECK(inp >= 0 && inp < nn, "node " << i << " has bad input " << inp);
      g.nodes[inp].outputs.push_back(i);
    }
    for (int v : n.vars) LTB_CHECK(v >= 0 && v < nv, "bad var ref " << v);
    for (auto& o : n.order)
      LTB_CHECK(o.first >= 0 && o.first < nv, "bad var in order " << o.first);
  }
  for (int i : g.inputs)
    LTB_CHECK(i >= 0 && i < nn && g.nodes[i].op == Op::read,
              "IR input " << i << " is not a read node");
  for (int o : g.outputs)
    LTB_CHECK(o >= 0 && o < nn && g.nodes[o].op == Op::write,
              "IR output " << o << " is not a write node");
  infer_var_sizes(g);
  return g;
}

void infer_var_sizes(IRGraph& g) {
  // compile.cpp:62-120: size() constraints first, then loop orders
  // (outer*inner+tail products) raise them.
  auto& vs = g.var_sizes;
  for (auto& n : g.nodes) {
    for (auto& c : n.constraints) {
      if (c.lhs->op != EOp::size) continue;
      auto r = ex_simplify(c.rhs);
      int64_t v;
      if (ex_is_val(r, &v)) vs[c.lhs->var] = v;
    }
    std::unordered_map<int, int64_t> tmp;
    for (auto it = n.order.rbegin(); it != n.order.rend(); ++it) {
      auto& t = tmp.emplace(it->first, 1).first->second;
      t = t * it->second.size + it->second.tail;
    }
    for (auto& p : tmp) {
      auto f = vs.find(p.first);
      vs[p.first] = f == vs.end() ? p.second : std::max(f->second, p.second);
    }
  }
  // second chance: size constraints whose rhs names other sizes
  for (int pass = 0; pass < 8; ++pass) {
    bool changed = false;
    for (auto& n : g.nodes)
      for (auto& c : n.constraints) {
        if (c.lhs->op != EOp::size || vs.count(c.lhs->var)) continue;
        int64_t v;
        if (ex_eval(ex_reify_sizes(c.rhs, vs), {}, &v)) {
          vs[c.lhs->var] = v;
          changed = true;
        }
      }
    if (!changed) break;
  }
  for (int v = 0; v < (int)g.var_names.size(); ++v)
    LTB_CHECK(vs.count(v), "size could not be deduced for var "
                               << g.var_names[v]);
}

std::vector<int> IRGraph::reduction_vars(int n) const {
  std::vector<int> out;
  const auto& node = nodes[n];
  for (int inp : node.inputs)
    for (int v : nodes[inp].vars)
      if (std::find(node.vars.begin(), node.vars.end(), v) == node.vars.end() &&
          std::find(out.begin(), out.end(), v) == out.end())
        out.push_back(v);
  return out;
}

std::vector<int> IRGraph::all_vars(int n) const {
  std::vector<int> out = nodes[n].vars;
  for (int inp : nodes[n].inputs)
    for (int v : nodes[inp].vars)
      if (std::find(out.begin(), out.end(), v) == out.end()) out.push_back(v);
  std::sort(out.begin(), out.end());
  return out;
}

// Restatement of IR::view_reduction_vars (ir.cpp:146-204), reduced to the
// question the index derivation asks: "is this view many-to-one?".
bool IRGraph::view_has_reduction(int n) const {
  const auto& node = nodes[n];
  auto is_out = [&](int v) {
    return std::find(node.vars.begin(), node.vars.end(), v) != node.vars.end();
  };
  std::vector<int> rhs_syms;
  for (auto& c : node.constraints) {
    if (c.lhs->op != EOp::var || !is_out(c.lhs->var)) continue;
    std::vector<int> vs;
    ex_vars(c.rhs, vs, true);
    for (int v : vs)
      if (!is_out(v) && std::find(rhs_syms.begin(), rhs_syms.end(), v) ==
                            rhs_syms.end())
        rhs_syms.push_back(v);
  }
  for (auto& c : node.constraints) {
    if (c.lhs->op != EOp::var || !is_out(c.lhs->var)) continue;
    std::vector<std::pair<int, ExP>> strides;
    for (int s : rhs_syms) strides.push_back({s, ex_simplify(ex_diff(c.rhs, s))});
    for (size_t k = 0; k < rhs_syms.size(); ++k) {
      int s = rhs_syms[k];
      int contiguous = 0;
      std::vector<std::pair<int, ExP>> rest;
      for (auto& p : strides) {
        float f;
        if (ex_eval_float(p.second, &f) && f <= 1)
          contiguous++;
        else
          rest.push_back(p);
      }
      for (auto& p : rest)
        if (ex_contains(p.second, s))
          p.second = ex_simplify(ex_bin(EOp::divide, p.second, ex_size(s)));
      strides = rest;
      if (contiguous > 1) return true;
    }
    if (strides.size() > 1) return true;
  }
  return false;
}

std::vector<int> topo_order(const IRGraph& g) {
  const int nn = (int)g.nodes.size();
  std::vector<int> indeg(nn, 0), out;
  for (int i = 0; i < nn; ++i) indeg[i] = (int)g.nodes[i].inputs.size();
  std::set<int> ready;
  for (int i = 0; i < nn; ++i)
    if (!indeg[i]) ready.insert(i);
  while (!ready.empty()) {
    int n = *ready.begin();
    ready.erase(ready.begin());
    out.push_back(n);
    for (int c : g.nodes[n].outputs)
      if (--indeg[c] == 0) ready.insert(c);
  }
  LTB_CHECK((int)out.size() == nn, "IR graph has a cycle");
  return out;
}

}  // namespace ltb
