// Oracle harness: drives the reference loop_tool CPU library (built from the
// reference sources by oracle/Makefile).  Test infrastructure only.
//
//   lt_ref_harness ir <program> <int params...>
//       Builds <program> with the reference lazy frontend (lazy.h) at the given
//       sizes and prints serialize(tensor.ir()) (serialization.cpp:175-237),
//       i.e. exactly the IR + default schedule the reference hands to
//       Backend::compile (lazy.cpp:430-438).
//   lt_ref_harness run <ir_file> <backend> <in_dir> <out_dir> [reps]
//       deserialize (serialization.cpp:239-332) -> LoopTree (ir.cpp:531) ->
//       getBackends().at(backend)->compile(lt) -> Compiled::run, reading
//       in_dir/in<i>.f32 and writing out_dir/out<j>.f32.  With reps > 0 the
//       run is repeated and per-run wall times are printed as JSON.
//   lt_ref_harness lazyrun <out_dir> <in_dir> <program> <int params...>
//       Runs <program> through the lazy frontend itself (TensorImpl::data,
//       lazy.h:219-260) with the default "cpp" backend: inputs are bound in
//       getInputBuffers order (lazy.cpp:72-88), no serialize round trip.
//   lt_ref_harness subtree <out_dir> <in_dir> <depth>[:backend] <program> <params...>
//       Annotates the first loop at <depth> with "[cuda]" (or "[backend]") and runs the tree
//       through the "cpu_interpreted" backend, which compiles that subtree
//       with the "cuda" backend and calls it per enclosing iteration.
//   lt_ref_harness fuzz <out_dir> <in_dir> <seed> <permute> <backend> <program> <params...>
//       Gives every non-view node of <program>'s IR a random schedule the
//       way the reference's own randomized test does (test/test.py:56-96
//       rand_split / rand_sched: each loop var split into up to 3 loops
//       with random factors and tails), and with <permute> = 1 also
//       shuffles the order of the var groups (the schedule is a function
//       of the seed).  Writes the scheduled IR (serialize) to out_dir/ir.txt
//       and, unless <backend> is "none", that backend's outputs on the
//       in-memory loop tree to out_dir/<backend><j>.f32.
//   lt_ref_harness annotate <depth> <annotation> <program> <params...>
//       Annotates the first loop at <depth> of <program>'s loop tree with
//       <annotation> through the reference's own annotate()
//       (mutate.cpp:694-712) and prints serialize() of the result.
//   lt_ref_harness lazytime <reps> <program> <params...>
//       Times the reference lazy frontend itself on <program>: leaves are
//       filled with seeded uniform values, one untimed T.data() compiles and
//       runs, then <reps> times force_recompute() + data() (lazy.h:219-260:
//       a fresh output allocation on the default hardware, Compiled::run
//       with sync, the result readable on the host) with the first and last
//       output element read on the host; prints {"seconds": [...]} (steady
//       clock, per call).  With LT_PLUGIN the default backend and hardware
//       are the plugin's "cuda".
//   lt_ref_harness tree <ir_file>      LoopTree::dump of the IR
//   lt_ref_harness code <ir_file>      the C the "cpp" backend generates
//   lt_ref_harness sizes <ir_file>     element counts of every I/O buffer
#include <loop_tool/cpp.h>
#include <loop_tool/loop_tool.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <random>
#include <cstdio>
#include <fstream>
#include <thread>
#include <unordered_set>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

namespace lz = loop_tool::lazy;
using loop_tool::Operation;
using lz::Constraint;
using lz::Expr;
using lz::Symbol;
using lz::Tensor;

static int64_t P(const std::vector<int64_t>& p, size_t i) {
  if (i >= p.size()) {
    std::cerr << "missing parameter #" << i << "\n";
    std::exit(2);
  }
  return p[i];
}

// python/nn.py:87-93 pad(), applied to one symbol
static Tensor pad_dim(const Tensor& X, const Symbol& s, int64_t pre,
                      int64_t post) {
  return X.pad(s, pre, post);
}

// python/nn.py:96-109 conv(): view X with sp = stride*sp_o + k, then
// (X * W).sum(channels shared with W, window dims)
static Tensor conv_like_python(Tensor X, Tensor W,
                               const std::vector<Symbol>& spatial,
                               const std::vector<Symbol>& window,
                               int64_t stride) {
  std::vector<Symbol> new_spatial;
  for (auto& s : spatial) new_spatial.emplace_back(Symbol(s.name() + "o"));
  std::vector<Symbol> outer;
  for (auto& d : X.shape()) {
    bool is_sp = false;
    for (auto& s : spatial) is_sp |= (s == d);
    if (!is_sp) outer.emplace_back(d);
  }
  std::vector<Constraint> cs;
  for (size_t i = 0; i < spatial.size(); ++i) {
    cs.emplace_back(Expr(spatial[i]),
                    Expr(stride) * Expr(new_spatial[i]) + Expr(window[i]));
  }
  std::vector<Symbol> view_shape = outer;
  view_shape.insert(view_shape.end(), new_spatial.begin(), new_spatial.end());
  view_shape.insert(view_shape.end(), window.begin(), window.end());
  X = X.to(view_shape, cs);
  std::vector<Symbol> red;
  for (auto& d : X.shape()) {
    bool in_w = false;
    for (auto& w : W.shape()) in_w |= (w == d);
    bool in_win = false;
    for (auto& w : window) in_win |= (w == d);
    if (in_w || in_win) red.emplace_back(d);
  }
  return (X * W).sum(red);
}

static Tensor build(const std::string& prog, const std::vector<int64_t>& p) {
  if (prog == "add" || prog == "sub" || prog == "mul" || prog == "div" ||
      prog == "min" || prog == "max") {
    Symbol N("N");
    Tensor A(P(p, 0)), B(P(p, 0));
    auto a = A.as(N), b = B.as(N);
    if (prog == "add") return a + b;
    if (prog == "sub") return a - b;
    if (prog == "mul") return a * b;
    if (prog == "div") return a / b;
    if (prog == "min") return a.min(b);
    return a.max(b);
  }
  if (prog == "exp" || prog == "sqrt" || prog == "neg" || prog == "recip" ||
      prog == "abs") {
    Symbol N("N");
    Tensor A(P(p, 0));
    auto a = A.as(N);
    if (prog == "exp") return a.exp();
    if (prog == "sqrt") return a.sqrt();
    if (prog == "neg") return -a;
    if (prog == "recip") return a.reciprocal();
    return a.abs();
  }
  if (prog == "chain") {  // a fused elementwise tree over three inputs
    Symbol N("N");
    Tensor A(P(p, 0)), B(P(p, 0)), C(P(p, 0));
    auto a = A.as(N), b = B.as(N), c = C.as(N);
    auto t = a * b + c;
    return ((t * t).sqrt() / (-a)).max(c) - b.reciprocal();
  }
  if (prog == "mm") {  // (A.to(m,k) * B.to(k,n)).sum(k)
    Symbol M("m"), K("k"), N("n");
    Tensor A(P(p, 0), P(p, 1)), B(P(p, 1), P(p, 2));
    return (A.as(M, K) * B.as(K, N)).sum(K);
  }
  if (prog == "bmm") {  // batched: (A[b,m,k] * B[b,k,n]).sum(k)
    Symbol Bs("b"), M("m"), K("k"), N("n");
    Tensor A(P(p, 0), P(p, 1), P(p, 2)), B(P(p, 0), P(p, 2), P(p, 3));
    return (A.as(Bs, M, K) * B.as(Bs, K, N)).sum(K);
  }
  if (prog == "softmax") {  // max over n, subtract, exp, sum over n, divide
    Symbol R("r"), N("n");
    Tensor X(P(p, 0), P(p, 1));
    auto x = X.as(R, N);
    auto mx = x.max(std::vector<Symbol>{N});
    auto e = (x - mx).exp();
    auto s = e.sum(N);
    return e / s;
  }
  if (prog == "rowsum" || prog == "rowmax" || prog == "colsum" ||
      prog == "colmax" || prog == "fullsum" || prog == "rowmin") {
    Symbol R("r"), N("n");
    Tensor X(P(p, 0), P(p, 1));
    auto x = X.as(R, N);
    if (prog == "rowsum") return x.sum(N);
    if (prog == "rowmax") return x.max(std::vector<Symbol>{N});
    if (prog == "rowmin") return x.min(std::vector<Symbol>{N});
    if (prog == "colsum") return x.sum(R);
    if (prog == "colmax") return x.max(std::vector<Symbol>{R});
    return x.sum(R, N);
  }
  if (prog == "maxpool") {  // nn.cpp:48-76 maxpool(X, {h,w}, k, stride)
    Symbol Nn("n"), C("c"), H("h"), W("w");
    Tensor X(P(p, 0), P(p, 1), P(p, 2), P(p, 3));
    return loop_tool::nn::maxpool(X.as(Nn, C, H, W), {H, W}, (int)P(p, 4),
                                  (int)P(p, 5));
  }
  if (prog == "conv") {  // N C H W CO K pad stride
    Symbol Nn("n"), C("c"), H("h"), W("w"), CO("co"), KH("kh"), KW("kw");
    Tensor X(P(p, 0), P(p, 1), P(p, 2), P(p, 3));
    Tensor Wt(P(p, 4), P(p, 1), P(p, 5), P(p, 5));
    auto x = X.as(Nn, C, H, W);
    int64_t pad = P(p, 6);
    std::vector<Symbol> spatial = {H, W};
    if (pad > 0) {
      x = pad_dim(x, H, pad, pad);
      x = pad_dim(x, x.shape()[3], pad, pad);
      spatial = {x.shape()[2], x.shape()[3]};
    }
    return conv_like_python(x, Wt.as(CO, C, KH, KW), spatial, {KH, KW},
                            P(p, 7));
  }
  if (prog == "conv1d") {  // test_lazy.cpp:302-330 LazyConv
    Symbol N("N"), No("No"), K("K");
    Tensor A(P(p, 0)), Wt(P(p, 1));
    auto X = A.as(N).to({No, K}, Constraint(N, No + K));
    return (X * Wt.as(K)).sum(K);
  }
  if (prog == "padconv1d") {  // test_cpp.cpp:136-160 CppView
    Symbol N("n"), Np("np"), No("no"), K("k");
    Tensor A(P(p, 0)), Wt(P(p, 1));
    auto X_pad = A.as(N).pad(N, P(p, 2)).as(Np);
    return (X_pad.to({No, K}, Constraint(Np, No + K)) * Wt.as(K)).sum(K);
  }
  if (prog == "pad1d") {  // test_lazy.cpp:416-434 LazyPadOnly
    Symbol N("N");
    Tensor X(P(p, 0));
    return X.as(N).pad(N, P(p, 1), P(p, 2));
  }
  if (prog == "pad2d") {  // test_views.py:6-16 test_pad
    Symbol M("m"), N("n");
    Tensor X(P(p, 0), P(p, 1));
    return X.as(M, N).pad(N, P(p, 2));
  }
  if (prog == "concat1d") {  // test_lazy.cpp:356-387
    Symbol N("N"), M("M");
    Tensor A(P(p, 0)), B(P(p, 1));
    return A.as(N) | B.as(M);
  }
  if (prog == "concat2d") {  // test_lazy.cpp:389-414
    Symbol N("N"), M0("M0"), M1("M1");
    Tensor A(P(p, 0), P(p, 1)), B(P(p, 0), P(p, 2));
    return A.as(N, M0) | B.as(N, M1);
  }
  if (prog == "transpose_flatten") {  // test_lazy.cpp:258-282 LazyTranspose
    Symbol M("M"), N("N"), K("K");
    Tensor A(P(p, 0), P(p, 1));
    auto a = A.as(M, N);
    return a.to({K}, Constraint(K, N * Expr::size(M) + M));
  }
  if (prog == "flatten") {  // test_lazy.cpp:284-300 LazyFlatten
    Symbol M("M"), N("N"), K("K");
    Tensor A(P(p, 0), P(p, 1));
    return A.as(M, N).flatten({M, N}, K);
  }
  if (prog == "transpose") {  // B[n,m] = A[m,n]
    Symbol M("M"), N("N");
    Tensor A(P(p, 0), P(p, 1));
    return A.as(M, N).to({N, M});
  }
  if (prog == "scale") {  // test_lazy.cpp:221-242 D = B * S (broadcast)
    Tensor B(P(p, 0)), S(1);
    Symbol N("N"), O("O");
    return B.as(N) * S.as(O);
  }
  if (prog == "bcast_add") {  // x[r,n] + b[n]
    Symbol R("r"), N("n");
    Tensor X(P(p, 0), P(p, 1)), Bv(P(p, 1));
    return X.as(R, N) + Bv.as(N);
  }
  if (prog == "mean_rows") {  // x.sum(n) / count  (python/nn.py mean idiom)
    Symbol R("r"), N("n");
    Tensor X(P(p, 0), P(p, 1)), One(P(p, 1));
    return X.as(R, N).sum(N) / One.as(N).sum(N);
  }
  if (prog == "layernorm") {  // (x - mean) / sqrt(var + eps), eps as input
    Symbol R("r"), N("n"), E("e");
    Tensor X(P(p, 0), P(p, 1)), Cnt(1), Eps(1);
    auto x = X.as(R, N);
    auto mean = x.sum(N) / Cnt.as(E);
    auto d = x - mean;
    auto var = (d * d).sum(N) / Cnt.as(E);
    return d / (var + Eps.as(E)).sqrt();
  }
  std::cerr << "unknown program " << prog << "\n";
  std::exit(2);
}

// test/test.py:56-82: the total size of a split list, one split, and up
// to `attempts` random splits of a (size, tail) loop list
using Splits = std::vector<std::pair<int64_t, int64_t>>;
static int64_t split_total(const Splits& s) {
  int64_t running = 1;
  for (auto it = s.rbegin(); it != s.rend(); ++it) running = it->first * running + it->second;
  return running;
}
static Splits do_split(const Splits& s, size_t idx, std::pair<int64_t, int64_t> ns) {
  Splits inner(s.begin() + idx + 1, s.end());
  const int64_t inner_size = split_total(inner);
  const int64_t outer_size = s[idx].first * inner_size + s[idx].second;
  const int64_t new_total = ns.first * inner_size + ns.second;
  Splits out(s.begin(), s.begin() + idx);
  out.push_back({outer_size / new_total, outer_size % new_total});
  out.push_back(ns);
  out.insert(out.end(), inner.begin(), inner.end());
  return out;
}
static Splits rand_split(Splits s, int attempts, std::mt19937_64& rng) {
  for (int a = 0; a < attempts; ++a) {
    const size_t idx = std::uniform_int_distribution<size_t>(0, s.size() - 1)(rng);
    const int64_t hi = (int64_t)std::sqrt((double)s[idx].first);
    if (hi < 2) continue;
    const int64_t f = std::uniform_int_distribution<int64_t>(2, hi)(rng);
    s = do_split(s, idx, {f, 0});
  }
  return s;
}

static std::string read_file(const std::string& path) {
  std::ifstream f(path);
  std::stringstream ss;
  ss << f.rdbuf();
  return ss.str();
}

int main(int argc, char** argv) {
  // LT_PLUGIN=<backend plugin .so>: load it (backend.cpp:63-65) and make its
  // "cuda" backend and hardware the defaults, as a user switching backends
  // would (backend.cpp:53-61, hardware.cpp:61).
  if (const char* plugin = std::getenv("LT_PLUGIN")) {
    try {
      loop_tool::loadLibrary(plugin);
      loop_tool::setDefaultBackend("cuda");
      for (auto& hw : loop_tool::getHardware())
        if (hw->name() == "cuda") loop_tool::setDefaultHardwareId(hw->id());
    } catch (const std::exception& e) {
      std::cerr << "plugin error: " << e.what() << "\n";
      return 5;
    }
  }
  if (argc < 3) {
    std::cerr << "usage: lt_ref_harness ir|run|tree|code|sizes ...\n";
    return 2;
  }
  std::string mode = argv[1];
  try {
    if (mode == "ir") {
      std::vector<int64_t> params;
      for (int i = 3; i < argc; ++i) params.emplace_back(std::stoll(argv[i]));
      auto T = build(argv[2], params);
      std::cout << loop_tool::serialize(T.ir());
      return 0;
    }
    if (mode == "lazyrun") {
      std::string out_dir = argv[2], in_dir = argv[3];
      std::vector<int64_t> params;
      for (int i = 5; i < argc; ++i) params.emplace_back(std::stoll(argv[i]));
      auto T = build(argv[4], params);
      auto tir = T.ir();
      loop_tool::LoopTree tlt(tir);
      loop_tool::Compiler tc(tlt);
      auto tsizes = tc.memory_sizes(true);
      std::unordered_set<const loop_tool::lazy::TensorImpl*> seen;
      auto leaves = T.impl()->getInputBuffers(seen);
      if (leaves.size() != tir.inputs().size()) {
        std::cerr << "leaf/input count mismatch\n";
        return 3;
      }
      for (size_t i = 0; i < leaves.size(); ++i) {
        auto path = in_dir + "/in" + std::to_string(i) + ".f32";
        std::ifstream f(path, std::ios::binary);
        f.read(reinterpret_cast<char*>(leaves[i]), tsizes[i] * sizeof(float));
        if ((size_t)f.gcount() != tsizes[i] * sizeof(float)) {
          std::cerr << "short input " << path << "\n";
          return 3;
        }
      }
      const float* out = T.data<float>();
      std::ofstream f(out_dir + "/out0.f32", std::ios::binary);
      f.write(reinterpret_cast<const char*>(out),
              tsizes[tir.inputs().size()] * sizeof(float));
      return 0;
    }
    if (mode == "lazytime") {
      const int reps = std::stoi(argv[2]);
      std::vector<int64_t> params;
      for (int i = 4; i < argc; ++i) params.emplace_back(std::stoll(argv[i]));
      auto T = build(argv[3], params);
      auto tir = T.ir();
      loop_tool::LoopTree tlt(tir);
      loop_tool::Compiler tc(tlt);
      auto tsizes = tc.memory_sizes(true);
      std::unordered_set<const loop_tool::lazy::TensorImpl*> seen;
      auto leaves = T.impl()->getInputBuffers(seen);
      uint64_t st = 0x9E3779B97F4A7C15ull;  // xorshift64: seeded uniform [-1, 1)
      for (size_t i = 0; i < leaves.size(); ++i) {
        float* f = static_cast<float*>(leaves[i]);
        for (int64_t e = 0; e < tsizes[i]; ++e) {
          st ^= st << 13;
          st ^= st >> 7;
          st ^= st << 17;
          f[e] = (float)((int64_t)(st >> 40) - (1 << 23)) * (1.0f / (1 << 23));
        }
      }
      const int64_t nout = tsizes[tir.inputs().size()];
      volatile float sink = T.data<float>()[0];
      std::cout << "{\"seconds\": [";
      for (int r = 0; r < reps; ++r) {
        auto t0 = std::chrono::steady_clock::now();
        T.force_recompute();
        const float* out = T.data<float>();
        sink = out[0] + out[nout - 1];
        auto t1 = std::chrono::steady_clock::now();
        std::cout << (r ? ", " : "") << std::chrono::duration<double>(t1 - t0).count();
      }
      (void)sink;
      std::cout << "]}\n";
      return 0;
    }
    if (mode == "annotate") {
      const int depth = std::stoi(argv[2]);
      const std::string annot = argv[3];
      std::vector<int64_t> params;
      for (int i = 5; i < argc; ++i) params.emplace_back(std::stoll(argv[i]));
      auto T = build(argv[4], params);
      loop_tool::LoopTree base(T.ir());
      loop_tool::LoopTree::TreeRef target = -1;
      base.walk([&](loop_tool::LoopTree::TreeRef r, int d) {
        if (target < 0 && d == depth && base.kind(r) == loop_tool::LoopTree::LOOP) target = r;
      });
      if (target < 0) {
        std::cerr << "no loop at depth " << depth << "\n";
        return 3;
      }
      std::cout << loop_tool::serialize(loop_tool::annotate(base, target, annot).ir);
      return 0;
    }
    if (mode == "fuzz") {
      std::string out_dir = argv[2], in_dir = argv[3];
      std::mt19937_64 rng(std::stoull(argv[4]));
      const bool permute = std::atoi(argv[5]) != 0;
      const std::string fbe = argv[6];
      std::vector<int64_t> params;
      for (int i = 8; i < argc; ++i) params.emplace_back(std::stoll(argv[i]));
      auto T = build(argv[7], params);
      auto ir = T.ir();
      for (auto n : ir.nodes()) {
        if (ir.node(n).op() == loop_tool::Operation::view) continue;
        // the default order holds each loop var once at its full size
        std::vector<std::pair<int, loop_tool::IR::LoopSize>> order;
        std::vector<std::vector<std::pair<int, loop_tool::IR::LoopSize>>> groups;
        for (auto& o : ir.order(n)) {
          const int attempts = std::uniform_int_distribution<int>(1, 3)(rng);
          Splits sp = rand_split({{o.second.size, o.second.tail}}, attempts, rng);
          if (split_total(sp) != split_total({{o.second.size, o.second.tail}})) {
            std::cerr << "split bookkeeping error\n";
            return 3;
          }
          std::vector<std::pair<int, loop_tool::IR::LoopSize>> g;
          for (auto& p : sp) g.push_back({o.first, loop_tool::IR::LoopSize{p.first, p.second}});
          groups.push_back(g);
        }
        if (permute) std::shuffle(groups.begin(), groups.end(), rng);
        for (auto& g : groups) order.insert(order.end(), g.begin(), g.end());
        ir.set_order(n, order);
      }
      std::ofstream(out_dir + "/ir.txt") << loop_tool::serialize(ir);
      if (fbe == "none") return 0;
      loop_tool::LoopTree flt(ir);
      loop_tool::Compiler fc(flt);
      auto fsizes = fc.memory_sizes(true);
      const size_t n_in = ir.inputs().size(), n_out = ir.outputs().size();
      {
        const std::string be = fbe;
        std::vector<std::vector<float>> bufs(n_in + n_out);
        std::vector<void*> mem;
        for (size_t i = 0; i < n_in + n_out; ++i) {
          bufs[i].assign(std::max<int64_t>(fsizes[i], 1), 0.f);
          if (i < n_in) {
            std::ifstream f(in_dir + "/in" + std::to_string(i) + ".f32", std::ios::binary);
            f.read(reinterpret_cast<char*>(bufs[i].data()), bufs[i].size() * sizeof(float));
            if ((size_t)f.gcount() != bufs[i].size() * sizeof(float)) {
              std::cerr << "short input " << i << "\n";
              return 3;
            }
          }
          mem.emplace_back(bufs[i].data());
        }
        auto cc = loop_tool::getBackends().at(be)->compile(flt);
        cc->run(mem, true);
        for (size_t j = 0; j < n_out; ++j) {
          std::ofstream f(out_dir + "/" + be + std::to_string(j) + ".f32", std::ios::binary);
          f.write(reinterpret_cast<const char*>(bufs[n_in + j].data()),
                  bufs[n_in + j].size() * sizeof(float));
        }
      }
      return 0;
    }
    if (mode == "subtree") {
      // subtree <out_dir> <in_dir> <depth> <program> <params...>: annotate
      // the first loop at <depth> with "[cuda]" and run the tree through
      // the interpreter, which hands that subtree to the "cuda" backend
      // (compile.cpp:273-417); inputs in the IR's input order
      std::string out_dir = argv[2], in_dir = argv[3];
      // <depth> or <depth>:<backend> (default backend "cuda")
      const std::string da = argv[4];
      const int depth = std::stoi(da.substr(0, da.find(':')));
      const std::string sub_backend =
          da.find(':') == std::string::npos ? "cuda" : da.substr(da.find(':') + 1);
      std::vector<int64_t> params;
      for (int i = 6; i < argc; ++i) params.emplace_back(std::stoll(argv[i]));
      auto T = build(argv[5], params);
      loop_tool::LoopTree base(T.ir());
      loop_tool::LoopTree::TreeRef target = -1;
      base.walk([&](loop_tool::LoopTree::TreeRef r, int d) {
        if (target < 0 && d == depth && base.kind(r) == loop_tool::LoopTree::LOOP) target = r;
      });
      if (target < 0) {
        std::cerr << "no loop at depth " << depth << "\n";
        return 3;
      }
      auto alt = loop_tool::annotate(base, target, "[" + sub_backend + "]");
      loop_tool::Compiler comp(alt);
      auto sizes = comp.memory_sizes(true);
      const size_t n_in = alt.ir.inputs().size(), n_out = alt.ir.outputs().size();
      std::vector<std::vector<float>> bufs(n_in + n_out);
      std::vector<void*> mem;
      for (size_t i = 0; i < n_in + n_out; ++i) {
        bufs[i].assign(std::max<int64_t>(sizes[i], 1), 0.f);
        if (i < n_in) {
          std::ifstream f(in_dir + "/in" + std::to_string(i) + ".f32", std::ios::binary);
          f.read(reinterpret_cast<char*>(bufs[i].data()), bufs[i].size() * sizeof(float));
          if ((size_t)f.gcount() != bufs[i].size() * sizeof(float)) {
            std::cerr << "short input " << i << "\n";
            return 3;
          }
        }
        mem.emplace_back(bufs[i].data());
      }
      auto cc = loop_tool::getBackends().at("cpu_interpreted")->compile(alt);
      cc->run(mem, true);
      for (size_t j = 0; j < n_out; ++j) {
        std::ofstream f(out_dir + "/out" + std::to_string(j) + ".f32", std::ios::binary);
        f.write(reinterpret_cast<const char*>(bufs[n_in + j].data()),
                bufs[n_in + j].size() * sizeof(float));
      }
      return 0;
    }
    auto ir = loop_tool::deserialize(read_file(argv[2]));
    loop_tool::LoopTree lt(ir);
    if (mode == "tree") {
      std::cout << lt.dump();
      return 0;
    }
    if (mode == "code") {
      std::cout << loop_tool::CppCompiler(lt).gen_string();
      return 0;
    }
    loop_tool::Compiler analysis(lt);
    auto sizes = analysis.memory_sizes(true);
    size_t n_in = ir.inputs().size(), n_out = ir.outputs().size();
    if (mode == "sizes") {
      std::cout << "{\"inputs\": [";
      for (size_t i = 0; i < n_in; ++i)
        std::cout << (i ? ", " : "") << sizes[i];
      std::cout << "], \"outputs\": [";
      for (size_t j = 0; j < n_out; ++j)
        std::cout << (j ? ", " : "") << sizes[n_in + j];
      std::cout << "]}\n";
      return 0;
    }
    if (mode != "run" || argc < 6) {
      std::cerr << "bad mode/arguments\n";
      return 2;
    }
    std::string backend = argv[3], in_dir = argv[4], out_dir = argv[5];
    int reps = argc > 6 ? std::atoi(argv[6]) : 0;
    // optional start gate: after compiling and one untimed run, wait until
    // this file exists before the timed reps, so that several concurrently
    // started harness processes time their runs together
    std::string gate = argc > 7 ? argv[7] : "";
    std::vector<std::vector<float>> bufs(n_in + n_out);
    std::vector<void*> mem;
    for (size_t i = 0; i < n_in + n_out; ++i) {
      bufs[i].assign(std::max<int64_t>(sizes[i], 1), 0.f);
      if (i < n_in) {
        auto path = in_dir + "/in" + std::to_string(i) + ".f32";
        std::ifstream f(path, std::ios::binary);
        if (!f) {
          std::cerr << "missing " << path << "\n";
          return 3;
        }
        f.read(reinterpret_cast<char*>(bufs[i].data()),
               bufs[i].size() * sizeof(float));
        if ((size_t)f.gcount() != bufs[i].size() * sizeof(float)) {
          std::cerr << "short input " << path << " expected "
                    << bufs[i].size() << " floats\n";
          return 3;
        }
      }
      mem.emplace_back(bufs[i].data());
    }
    auto cc = loop_tool::getBackends().at(backend)->compile(lt);
    cc->run(mem, true);
    if (!gate.empty()) {
      std::ofstream(out_dir + "/ready").put('1');
      for (int w = 0; w < 600000 && !std::ifstream(gate); ++w)  // at most 10 minutes
        std::this_thread::sleep_for(std::chrono::milliseconds(1));
    }
    if (reps > 0) {
      std::cout << "{\"seconds\": [";
      for (int r = 0; r < reps; ++r) {
        auto t0 = std::chrono::steady_clock::now();
        cc->run(mem, true);
        auto t1 = std::chrono::steady_clock::now();
        std::cout << (r ? ", " : "")
                  << std::chrono::duration<double>(t1 - t0).count();
      }
      std::cout << "]}\n";
    }
    for (size_t j = 0; j < n_out; ++j) {
      auto path = out_dir + "/out" + std::to_string(j) + ".f32";
      std::ofstream f(path, std::ios::binary);
      f.write(reinterpret_cast<const char*>(bufs[n_in + j].data()),
              bufs[n_in + j].size() * sizeof(float));
    }
    return 0;
  } catch (const std::exception& e) {
    std::cerr << "reference error: " << e.what() << "\n";
    return 4;
  }
}
