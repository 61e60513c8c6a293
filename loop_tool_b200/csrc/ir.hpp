// IR model for the B200 backend: the reference's serialized IR text
// (serialization.cpp:175-237 writes it, :239-332 reads it) parsed into a
// dataflow graph whose index expressions are written over IR variables.
//
// Symbols never outlive the parse: every symbol in a view constraint is
// replaced by the IR variable the node's sym->var map binds it to (the
// reference keeps one symbol per variable too, compile.cpp:62-80), so
// expressions here are trees over variable ids.
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

namespace ltb {

struct Error : std::runtime_error {
  using std::runtime_error::runtime_error;
};

#define LTB_CHECK(cond, msg)                                        \
  do {                                                              \
    if (!(cond)) {                                                  \
      std::ostringstream _ltb_ss;                                   \
      _ltb_ss << msg << " [" << __FILE__ << ":" << __LINE__ << "]"; \
      throw ::ltb::Error(_ltb_ss.str());                            \
    }                                                               \
  } while (0)

// Operation codes, numbered exactly as the reference's OPS(_) list
// (ir.h:21-39) because the serialized text stores them as integers.
enum class Op : int32_t {
  constant = 0,
  write,
  read,
  view,
  copy,
  add,
  subtract,
  multiply,
  divide,
  min,
  max,
  log,
  exp,
  sqrt,
  abs,
  negate,
  reciprocal,
  name
};
const char* op_name(Op op);

// ---------------------------------------------------------------- symbolic
// Expression ops numbered as the reference's symbolic::Op (symbolic.h:38-50).
enum class EOp : int32_t {
  value = -1,  // leaf constant (not an Op in the reference)
  var = -2,    // leaf variable
  negate = 1,
  reciprocal = 2,
  size = 3,
  max = 4,
  add = 5,
  multiply = 6,
  divide = 7,
  modulo = 8
};

struct Ex;
using ExP = std::shared_ptr<const Ex>;
struct Ex {
  EOp op;
  int64_t val = 0;  // value leaf
  int var = -1;     // var leaf, or the argument var of size()
  ExP a, b;
};

ExP ex_val(int64_t v);
ExP ex_var(int v);
ExP ex_size(int v);
ExP ex_un(EOp op, ExP a);
ExP ex_bin(EOp op, ExP a, ExP b);

bool ex_is_val(const ExP& e, int64_t* v = nullptr);
bool ex_equal(const ExP& x, const ExP& y);
// vars that occur outside size() (the reference's symbols(false))
void ex_vars(const ExP& e, std::vector<int>& out, bool include_sized = false);
bool ex_contains(const ExP& e, int var);
ExP ex_replace_var(const ExP& e, int var, const ExP& with);
ExP ex_reify_sizes(const ExP& e, const std::unordered_map<int, int64_t>& sz);
// Folding/identity rules that keep C int64 semantics (trunc division).
ExP ex_simplify(const ExP& e);
// d e / d var for sums/products/quotients (symbolic.cpp:907-962 rules)
ExP ex_diff(const ExP& e, int var);
// Evaluate with every var bound; returns false if a var is unbound.
bool ex_eval(const ExP& e, const std::unordered_map<int, int64_t>& env,
             int64_t* out);
// Constant-only evaluation in the reference's float arithmetic
// (symbolic.cpp:305-353): used only where the reference itself compares a
// float-evaluated quantity (the bijective-view modulus).
bool ex_eval_float(const ExP& e, float* out);
// Inclusive range of e when every var v ranges over [0, size(v)-1].
bool ex_range(const ExP& e, const std::unordered_map<int, int64_t>& sz,
              int64_t* lo, int64_t* hi);
std::string ex_str(const ExP& e, const std::vector<std::string>* names = nullptr);

// -------------------------------------------------------------------- IR
struct LoopSize {
  int64_t size;
  int64_t tail;
};

struct Constraint {
  ExP lhs, rhs;
};

struct Node {
  Op op;
  std::vector<int> inputs;
  std::vector<int> vars;
  std::vector<Constraint> constraints;
  float priority = 0;
  std::vector<std::pair<int, LoopSize>> order;
  std::vector<int> reuse_disabled;
  std::vector<std::string> loop_annotations;
  std::string annotation;
  std::vector<int> outputs;  // consumers (filled after parsing)
};

struct IRGraph {
  std::vector<std::string> var_names;
  std::vector<Node> nodes;
  std::vector<int> inputs;
  std::vector<int> outputs;
  std::unordered_map<int, int64_t> var_sizes;

  std::vector<int> reduction_vars(int n) const;  // ir.cpp:206-221
  std::vector<int> all_vars(int n) const;        // ir.cpp:223-239
  bool view_has_reduction(int n) const;          // ir.cpp:146-204
};

// Parse the reference's serialized IR text.  Throws ltb::Error.
IRGraph parse_ir(const std::string& text);
// Variable sizes: size() constraints and loop orders (compile.cpp:62-120).
void infer_var_sizes(IRGraph& g);
// Topological order by dependencies (ties by node id).
std::vector<int> topo_order(const IRGraph& g);

}  // namespace ltb
