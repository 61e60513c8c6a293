// C ABI of the B200 backend: compile (lower + upload), run (launch the plan
// on a stream), properties, and the "cuda" hardware allocator.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <limits>
#include <map>
#include <mutex>
#include <queue>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/loop_tool_b200.h"
#include "kernels.h"
#include "lower.hpp"
#include "tc_api.h"

static_assert(sizeof(LtbStage) % 16 == 0, "stage descriptor must be 16B-sized");

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define CUDA_TRY(expr)                                                     \
  do {                                                                     \
    cudaError_t _e = (expr);                                               \
    if (_e != cudaSuccess)                                                 \
      throw CudaFailure(std::string(#expr) + ": " + cudaGetErrorString(_e)); \
  } while (0)

struct CudaFailure : std::runtime_error {
  using std::runtime_error::runtime_error;
};

ltb::LowerOptions parse_options(const char* s) {
  ltb::LowerOptions o;
  if (!s) return o;
  std::istringstream ss(s);
  for (std::string kv; std::getline(ss, kv, ';');) {
    auto p = kv.find('=');
    if (p == std::string::npos) continue;
    auto k = kv.substr(0, p), v = kv.substr(p + 1);
    if (k == "precision") {
      if (v == "fp32") o.precision = ltb::Precision::fp32;
      else if (v == "bf16") o.precision = ltb::Precision::bf16;
      else if (v == "bf16x3") o.precision = ltb::Precision::bf16x3;
      else if (v == "bf16x4") o.precision = ltb::Precision::bf16x4;
      else if (v == "bf16x6") o.precision = ltb::Precision::bf16x6;
      else throw ltb::Error("unknown precision '" + v + "'");
    } else if (k == "fuse_rows") {
      o.fuse_rows = v != "0";
    } else if (k == "tensor_cores") {
      o.use_tensor_cores = v != "0";
    } else if (k == "kahan_threshold") {
      o.kahan_threshold = std::stoi(v);
    } else {
      throw ltb::Error("unknown option '" + k + "'");
    }
  }
  return o;
}

struct GemmTables {
  int stage = -1;
  int64_t nbatch = 1;
  std::vector<int64_t> a_boff, b_boff, c_boff;  // per batch
  int64_t *a_row = nullptr, *a_k = nullptr, *b_row = nullptr, *b_k = nullptr;
  int64_t *c_row = nullptr, *c_col = nullptr;
  int32_t *ag_row = nullptr, *ag_k = nullptr, *ag_ub = nullptr;
  int32_t *bg_row = nullptr, *bg_k = nullptr, *bg_ub = nullptr;
  int a_ng = 0, b_ng = 0;
  bool a_dense = false, b_dense = false;
  int64_t a_ldr = 0, a_ldk = 0, b_ldr = 0, b_ldk = 0;
  // tensor-core path: packed K-major BF16 operands and their tensor maps
  bool tc = false;
  int nseg = 1, a_mask = 1, b_mask = 1;
  int64_t Kp = 0, tiles = 0;
  int a_slot = -1, b_slot = -1;       // scratch slots of the packed operands
  LtbTcProblem prob{};                // launch template (maps/c bound per run)
  bool a_kcontig = true, b_kcontig = true, unit_cols = false;
  // output rows crow[r] = c_row0 + r * c_ld with unit columns, ld and every
  // offset a multiple of 4 floats: written by TMA stores (LtbTcProblem::c_tma)
  bool c_tma = false;
  int64_t c_row0 = 0, c_ld = 0;
  bool a_off32 = false, b_off32 = false;  // operand offsets fit in int32
  bool a_k32 = false, b_k32 = false;      // k offsets alone fit in int32
  // implicit-GEMM convolution: A packed as NHWC BF16 image(s) read by 4-D
  // TMA boxes (LtbTcProblem::img); B's K order permuted to (kh, kw, c)
  bool img = false;
  int img_kinds = 1;                  // images in the A slot: hi (+ lo (+ lo2))
  int64_t img_elems = 0;              // elements of one image
  LtbImageJob ijob{};                 // base / hi / lo / lo2 bound at launch
  int bn = 256;                       // tensor-core tile width (128 or 256)
  int epi = 0;                        // 1: shared-memory transposed epilogue,
                                      // 2: two CTAs per SM, 3: halo image tiles,
                                      // 4: 256 x 256 tiles on CTA pairs,
                                      // 5: halo image tiles on CTA pairs
  // halo image tiles (single-segment image operands, N <= 128): the launch
  // template in halo geometry, valid when halo_ok
  LtbTcProblem halo{};
  bool halo_ok = false;
};

bool halo_form(int epi) { return epi == 3 || epi == 5; }

// Tile form of a tensor-core contraction: output tiles are 128 x bn, or
// 256 x 256 on CTA pairs (epi 4, plain operands); halo tiles (epi 3, 5) are
// the halo geometry's m-tiles.
void set_tile_n(GemmTables& t, int bn, int epi) {
  if (halo_form(epi) && !(t.halo_ok && bn == 128)) epi = 0;
  if (epi == 4 && (t.img || bn != 256)) epi = 0;
  t.bn = bn;
  t.epi = epi;
  if (!t.img) t.prob.tiles_m = (int)((t.prob.M + (epi == 4 ? 255 : 127)) / (epi == 4 ? 256 : 128));
  const int64_t tn = (t.prob.N + bn - 1) / bn;
  t.prob.tiles_n = (int)tn;
  t.tiles = halo_form(epi) ? (int64_t)t.halo.tiles_m : (int64_t)t.prob.tiles_m * tn;
}

// Launch variant of a tile form (ltb_launch_gemm_tc, schedules): tile
// width | form (133: halo tiles on CTA pairs), or 258 for CTA pairs.
int variant_code(const GemmTables& t) { return t.epi == 4 ? 258 : t.bn | t.epi; }

// Rows of a B' tensor-map box: the tile width, or half of it on CTA pairs.
int b_box_rows(const GemmTables& t) { return t.epi == 4 ? 128 : t.epi == 5 ? 64 : t.bn; }

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

// The image repack job of a run: the operand's buffer and the A slot, which
// holds the hi image, then the lo and lo2 images when the split has them.
LtbImageJob image_job(const GemmTables& t, const float* base, void* a_slot) {
  LtbImageJob j = t.ijob;
  j.base = base;
  j.hi = a_slot;
  char* const at = static_cast<char*>(a_slot);
  j.lo = t.img_kinds >= 2 ? at + t.img_elems * 2 : nullptr;
  j.lo2 = t.img_kinds == 3 ? at + t.img_elems * 4 : nullptr;
  return j;
}

// All of a compiled object's constant device data (stage descriptors,
// contraction offset tables, the timeout flag) in one allocation and one
// copy: pointers are recorded as (slot, offset) and patched at finalize.
struct Arena {
  std::vector<unsigned char> host;
  std::vector<std::pair<void**, size_t>> fix;
  template <typename T>
  void add(const std::vector<T>& v, T** slot) {
    *slot = nullptr;
    if (v.empty()) return;
    const size_t off = (host.size() + 255) / 256 * 256;
    host.resize(off + v.size() * sizeof(T));
    memcpy(host.data() + off, v.data(), v.size() * sizeof(T));
    fix.push_back({reinterpret_cast<void**>(slot), off});
  }
  void finalize(std::vector<void*>& owned) {
    if (host.empty()) return;
    void* base = nullptr;
    CUDA_TRY(cudaMalloc(&base, host.size()));
    owned.push_back(base);
    CUDA_TRY(cudaMemcpy(base, host.data(), host.size(), cudaMemcpyHostToDevice));
    for (auto& f : fix) *f.first = static_cast<unsigned char*>(base) + f.second;
  }
};

template <typename T>
T* upload(const std::vector<T>& v, std::vector<void*>& owned) {
  if (v.empty()) return nullptr;
  void* p = nullptr;
  CUDA_TRY(cudaMalloc(&p, v.size() * sizeof(T)));
  CUDA_TRY(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  owned.push_back(p);
  return static_cast<T*>(p);
}

}  // namespace

int ltb_set_last_error(int code, const char* msg) { return fail(code, msg); }

namespace {

// Timeout flags of the bounded waits, one per (device, stream).  A kernel
// whose wait gives up raises the flag of the stream it was launched on; the
// next synchronising call on that stream (ltb_run / ltb_graph_run with
// sync, ltb_synchronize, ltb_tune) reports LTB_ERR_TIMEOUT and clears it, so
// an asynchronous run's timeout is charged to its own stream, not to
// whichever run synchronises next.  Each device's table is one allocation,
// made when the first loop tree is compiled on it (never in a run); with
// more than kFlagSlots distinct streams on a device, later streams share
// slots (a timeout is then reported on every stream of its slot).
constexpr int kFlagSlots = 1024;
struct FlagTable {
  int* d = nullptr;
  std::map<uintptr_t, int> slot;
};
std::mutex g_flag_mu;
FlagTable g_flags[64];

void ensure_flag_table(int dev) {
  std::lock_guard<std::mutex> g(g_flag_mu);
  FlagTable& t = g_flags[dev];
  if (t.d) return;
  CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(&t.d), kFlagSlots * sizeof(int)));
  CUDA_TRY(cudaMemset(t.d, 0, kFlagSlots * sizeof(int)));
}

// the flag of stream st on device dev (its table exists)
int* timeout_flag(int dev, cudaStream_t st) {
  std::lock_guard<std::mutex> g(g_flag_mu);
  FlagTable& t = g_flags[dev];
  const uintptr_t key = reinterpret_cast<uintptr_t>(st);
  auto it = t.slot.find(key);
  if (it != t.slot.end()) return t.d + it->second;
  const int n = (int)t.slot.size();
  const int s = n < kFlagSlots ? n : (int)(key % kFlagSlots);
  t.slot[key] = s;
  return t.d + s;
}

// After stream st has been synchronised: true (and the flag cleared) if a
// bounded wait launched on it gave up.
bool take_timeout(int dev, cudaStream_t st) {
  {
    std::lock_guard<std::mutex> g(g_flag_mu);
    if (!g_flags[dev].d) return false;
  }
  int* f = timeout_flag(dev, st);
  int flag = 0;
  CUDA_TRY(cudaMemcpyAsync(&flag, f, sizeof(int), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  if (!flag) return false;
  CUDA_TRY(cudaMemsetAsync(f, 0, sizeof(int), st));
  CUDA_TRY(cudaStreamSynchronize(st));
  return true;
}

}  // namespace

struct ltb_compiled {
  std::string ir_text;
  ltb::IRGraph ir;
  ltb::Plan plan;
  ltb::LowerOptions opt;
  int device = 0;
  int sms = 148;
  LtbStage* d_stages = nullptr;
  std::vector<int> split_of;          // per stage split count
  std::vector<size_t> scratch_off;    // byte offsets within scratch block
  size_t scratch_bytes = 0;
  void* scratch = nullptr;            // default scratch block
  std::vector<GemmTables> gemms;      // per contraction stage
  std::vector<int> gemm_of;           // stage -> index into gemms (or -1)
  std::vector<void*> owned;           // device allocations to free
  std::mutex mu;                      // guards the default scratch block
  cudaEvent_t scratch_done = nullptr; // recorded after each run on the default scratch
  int64_t bandwidth_gbs = 0;
  int launches = 0;
  std::vector<LtbCfg> cfg;            // per stage launch schedule (autotuner)
  cudaStream_t aux = nullptr;         // second stream of pipelined host-buffer runs
  std::mutex aux_mu;
  uint64_t key = 0;                   // IR-text + options hash (schedule cache key)
  bool tuned = false;                 // schedules came from the tuner / cache
};

namespace {

int64_t stage_outs(const LtbStage& d) {
  int64_t o = 1;
  for (int k = 0; k < d.nout; ++k) o *= d.size[k];
  return o;
}

// A stride-1 2-D window over an NCHW-like operand: rows (n, ho, wo) or
// (ho, wo), k (c, kh, kw) in any order, x(n, c, ho + kh + off_h,
// wo + kw + off_w) with unit column stride, row pitch wx, channel pitch cs,
// zero outside [0, ub_h) x [0, ub_w) (padding guards) or no guards.
struct ImageGeom {
  int64_t nimg = 1, ns = 0, ho = 0, wo = 0, c = 0, kh = 0, kw = 0, wx = 0, cs = 0;
  int kh_dim = -1, kw_dim = -1, c_dim = -1;
  int off_h = 0, ub_h = 1 << 30, off_w = 0, ub_w = 1 << 30;
};

bool detect_image(const LtbStage& d, const LtbLoad& A, const std::vector<int>& md,
                  const std::vector<int>& kd, ImageGeom& g) {
  if (kd.size() != 3 || (md.size() != 2 && md.size() != 3) || A.nq) return false;
  const int wo = md.back(), ho = md[md.size() - 2];
  g.wx = A.coef[ho];
  if (A.coef[wo] != 1 || g.wx < 2) return false;
  for (int k : kd) {
    if (A.coef[k] == 1 && g.kw_dim < 0) g.kw_dim = k;
    else if (A.coef[k] == g.wx && g.kh_dim < 0) g.kh_dim = k;
    else g.c_dim = k;
  }
  if (g.kw_dim < 0 || g.kh_dim < 0 || g.c_dim < 0) return false;
  g.cs = A.coef[g.c_dim];
  g.c = d.size[g.c_dim];
  g.kh = d.size[g.kh_dim];
  g.kw = d.size[g.kw_dim];
  g.ho = d.size[ho];
  g.wo = d.size[wo];
  if (g.cs < 1 || g.c % 64 || g.wo % 8 || g.wo > 128) return false;
  if (md.size() == 3) {
    g.nimg = d.size[md[0]];
    g.ns = A.coef[md[0]];
  }
  if (A.ng == 0) return A.off == 0;
  if (A.ng != 2) return false;
  bool fh = false, fw = false;
  for (int q = A.g0; q < A.g0 + A.ng; ++q) {
    const LtbGuard& G = d.guards[q];
    for (int k = 0; k < d.ndim; ++k) {
      const bool on_h = k == ho || k == g.kh_dim, on_w = k == wo || k == g.kw_dim;
      const bool h_guard = G.coef[ho] == 1 && G.coef[g.kh_dim] == 1;
      if (G.coef[k] != ((h_guard ? on_h : on_w) ? 1 : 0)) return false;
    }
    if (G.off < -(1 << 20) || G.off > (1 << 20) || G.ub > (1 << 30)) return false;
    if (G.coef[ho] == 1) {
      fh = true;
      g.off_h = (int)G.off;
      g.ub_h = (int)G.ub;
    } else {
      fw = true;
      g.off_w = (int)G.off;
      g.ub_w = (int)G.ub;
    }
  }
  return fh && fw && A.off == (int64_t)g.off_h * g.wx + g.off_w;
}

// Split a contraction's affine operand loads into per-row / per-k tables.
void build_gemm(ltb_compiled* c, int si, GemmTables& t, Arena& ar) {
  const ltb::PlanStage& ps = c->plan.stages[si];
  const LtbStage& d = ps.dev;
  const ltb::Contraction& con = ps.con;
  auto dim_of = [&](int var) {
    auto it = std::find(ps.dim_vars.begin(), ps.dim_vars.end(), var);
    return (int)(it - ps.dim_vars.begin());
  };
  std::vector<int> bd, md, nd, kd;
  for (int v : con.bvars) bd.push_back(dim_of(v));
  for (int v : con.mvars) md.push_back(dim_of(v));
  for (int v : con.nvars) nd.push_back(dim_of(v));
  for (int v : con.kvars) kd.push_back(dim_of(v));
  // enumerate a role's coordinates row-major and evaluate coef . x
  auto table = [&](const std::vector<int>& dims, const int64_t* coef,
                   int64_t off) {
    int64_t n = 1;
    for (int k : dims) n *= d.size[k];
    std::vector<int64_t> out(n);
    std::vector<int64_t> x(dims.size(), 0);
    for (int64_t i = 0; i < n; ++i) {
      int64_t v = off;
      for (size_t q = 0; q < dims.size(); ++q) v += coef[dims[q]] * x[q];
      out[i] = v;
      for (int q = (int)dims.size() - 1; q >= 0; --q) {
        if (++x[q] < d.size[dims[q]]) break;
        x[q] = 0;
      }
    }
    return out;
  };
  const LtbLoad& A = d.loads[con.a_load];
  const LtbLoad& B = d.loads[con.b_load];
  for (int g = A.g0; g < A.g0 + A.ng; ++g)
    for (int k : bd)
      if (d.guards[g].coef[k]) throw ltb::Error("guard over batch dims");
  t.a_boff = table(bd, A.coef, 0);
  t.b_boff = table(bd, B.coef, 0);
  t.c_boff = table(bd, d.out_coef, 0);
  t.nbatch = (int64_t)t.a_boff.size();
  ar.add(table(md, A.coef, A.off), &t.a_row);
  ar.add(table(kd, A.coef, 0), &t.a_k);
  ar.add(table(nd, B.coef, B.off), &t.b_row);
  ar.add(table(kd, B.coef, 0), &t.b_k);
  ar.add(table(md, d.out_coef, d.out_off), &t.c_row);
  ar.add(table(nd, d.out_coef, 0), &t.c_col);
  auto guards = [&](const LtbLoad& L, const std::vector<int>& rd,
                    int32_t** grow, int32_t** gk, int32_t** gub, int* ng) {
    std::vector<int32_t> vr, vk, vu;
    for (int g = L.g0; g < L.g0 + L.ng; ++g) {
      const LtbGuard& G = d.guards[g];
      for (auto v : table(rd, G.coef, G.off)) vr.push_back((int32_t)v);
      for (auto v : table(kd, G.coef, 0)) vk.push_back((int32_t)v);
      vu.push_back((int32_t)G.ub);
    }
    *ng = L.ng;
    ar.add(vr, grow);
    ar.add(vk, gk);
    ar.add(vu, gub);
  };
  guards(A, md, &t.ag_row, &t.ag_k, &t.ag_ub, &t.a_ng);
  guards(B, nd, &t.bg_row, &t.bg_k, &t.bg_ub, &t.b_ng);

  auto ktab_a = table(kd, A.coef, 0), ktab_b = table(kd, B.coef, 0);
  // dense = offsets are an arithmetic progression in the flat row / k index
  auto arith = [](const std::vector<int64_t>& v, int64_t* step) {
    *step = v.size() > 1 ? v[1] - v[0] : 0;
    for (size_t i = 1; i < v.size(); ++i)
      if (v[i] - v[i - 1] != *step) return false;
    return true;
  };
  // packing orientation: the direction (k or rows) whose neighbouring
  // offsets are most often adjacent in memory gets the warp's lanes, e.g.
  // rows (output pixels) for an im2col operand, k for a row-major A
  auto unit_frac = [](const std::vector<int64_t>& v) {
    if (v.size() < 2) return 1.0;
    size_t u = 0;
    for (size_t i = 1; i < v.size(); ++i) u += v[i] - v[i - 1] == 1;
    return (double)u / (double)(v.size() - 1);
  };
  {
    auto ra = table(md, A.coef, A.off), rb = table(nd, B.coef, B.off);
    t.a_dense = A.ng == 0 && ra[0] == 0 && arith(ra, &t.a_ldr) && arith(ktab_a, &t.a_ldk);
    t.b_dense = B.ng == 0 && rb[0] == 0 && arith(rb, &t.b_ldr) && arith(ktab_b, &t.b_ldk);
    t.a_kcontig = unit_frac(ktab_a) >= unit_frac(ra);
    t.b_kcontig = unit_frac(ktab_b) >= unit_frac(rb);
    auto maxabs = [](const std::vector<int64_t>& v) {
      int64_t m = 0;
      for (auto x : v) m = std::max<int64_t>(m, x < 0 ? -x : x);
      return m;
    };
    const int64_t lim = int64_t(1) << 31;
    t.a_off32 = maxabs(ra) + maxabs(ktab_a) < lim;
    t.b_off32 = maxabs(rb) + maxabs(ktab_b) < lim;
    t.a_k32 = maxabs(ktab_a) < lim;
    t.b_k32 = maxabs(ktab_b) < lim;
  }
  auto ctab = table(nd, d.out_coef, 0);
  t.unit_cols = true;
  for (size_t j = 0; j < ctab.size(); ++j) t.unit_cols = t.unit_cols && ctab[j] == (int64_t)j;
  {
    auto rc = table(md, d.out_coef, d.out_off);
    int64_t ld = 0;
    const bool affine = arith(rc, &ld);
    if (rc.size() == 1) ld = (con.N + 3) / 4 * 4;  // one row: any pitch
    t.c_row0 = rc[0];
    t.c_ld = ld;
    t.c_tma = affine && t.unit_cols && ld >= con.N && ld % 4 == 0 && rc[0] >= 0 && rc[0] % 4 == 0;
    for (auto o : t.c_boff) t.c_tma = t.c_tma && o % 4 == 0;
  }
  if (c->opt.precision != ltb::Precision::fp32 && c->opt.use_tensor_cores &&
      con.M < (1LL << 31) && con.N < (1LL << 31)) {
    t.tc = true;
    // split-BF16 along K: bit s of a mask selects hi (1) or lo (0) for
    // segment s, bit 8 + s the third piece lo2.  bf16x3: A' = [Ah|Al|Ah],
    // B' = [Bh|Bh|Bl] (Al*Bl dropped); bf16x4 adds Al*Bl: A' = [Ah|Al|Ah|Al],
    // B' = [Bh|Bh|Bl|Bl]; bf16x6 (three pieces, FP32's whole significand):
    // A' = [Ah|Al|Ah|Al|Al2|Ah], B' = [Bh|Bh|Bl|Bl|Bh|Bl2].
    switch (c->opt.precision) {
      case ltb::Precision::bf16x3: t.nseg = 3; t.a_mask = 0x5; t.b_mask = 0x3; break;
      case ltb::Precision::bf16x4: t.nseg = 4; t.a_mask = 0x5; t.b_mask = 0x3; break;
      case ltb::Precision::bf16x6:
        t.nseg = 6;
        t.a_mask = 0x25 | (0x10 << 8);
        t.b_mask = 0x13 | (0x20 << 8);
        break;
      default: t.nseg = 1; t.a_mask = 0x1; t.b_mask = 0x1; break;
    }
    t.Kp = (t.nseg * con.K + 7) / 8 * 8;
    // packed BF16 operands live in the run's scratch (2 BF16 per float slot)
    auto& P = c->plan;
    t.a_slot = P.num_slots();
    P.scratch_elems.push_back((con.M * t.Kp + 1) / 2);
    t.b_slot = P.num_slots();
    P.scratch_elems.push_back((con.N * t.Kp + 1) / 2);
    const int tm = (int)((con.M + ltb_tc_tile_m() - 1) / ltb_tc_tile_m());
    LtbTcProblem& e = t.prob;
    e.map_a = e.map_b = nullptr;
    e.c = nullptr;
    // crow / ccol point into the arena, which is only placed at finalize:
    // bound at launch time
    e.crow = e.ccol = nullptr;
    e.Kp = t.Kp;
    e.tile_start = 0;
    e.M = (int)con.M;
    e.N = (int)con.N;
    e.tiles_m = tm;
    e.unit_cols = t.unit_cols ? 1 : 0;
    e.c_tma = t.c_tma ? 1 : 0;  // and per run: C + c_row0 16-byte aligned
    e.map_c = nullptr;
    // the six-product mode drains every 2 k blocks (128 K): its pieces
    // carry FP32's whole significand, so the accumulation's truncation is
    // what is left to bound; plain BF16 accumulates the whole K in TMEM
    // (its inputs' rounding, 2^-9 of each product, outweighs the
    // truncation, ~2^-24 a K=16 step), so a tile is drained once
    e.chunk_blocks = t.nseg >= 6 ? 2 : t.nseg == 1 ? (int)((t.Kp + 63) / 64) : 0;
    // ... only within its main segment (Ah * Bh, the first K of the packed
    // K): the five correction segments' products are 2^-8 of those, so
    // 512-K chunks truncate them no more than the main segment's 128-K
    // chunks (a CPU model of the arithmetic: the same error, fewer drains);
    // ×3 / ×4, whose error is that of the products they drop, keep 512-K
    // chunks on the main segment and drain their corrections every 4096 K
    e.main_blocks = t.nseg >= 3 ? (int)((con.K + 63) / 64) : 0;
    e.rest_blocks = t.nseg >= 6 ? 8 : t.nseg >= 3 ? 64 : 0;
    ImageGeom ig;
    if (t.nbatch == 1 && t.Kp == t.nseg * con.K && detect_image(d, A, md, kd, ig)) {
      // implicit GEMM: A' never materialises; the A slot holds the padded
      // NHWC image(s), hi (+ lo for split modes, + lo2 for three-piece ones)
      t.img = true;
      t.c_tma = false;  // image tiles' rows are not one progression
      e.c_tma = 0;
      const int segs = (1 << t.nseg) - 1;
      t.img_kinds = ((t.a_mask >> 8) & segs) ? 3 : (~t.a_mask & segs) ? 2 : 1;
      const int64_t hp = ig.ho + ig.kh - 1, wp = ig.wo + ig.kw - 1;
      t.img_elems = ig.nimg * hp * wp * ig.c;
      P.scratch_elems[t.a_slot - (P.n_in + P.n_out)] = (t.img_kinds * t.img_elems + 1) / 2;
      LtbImageJob& j = t.ijob;
      j.off = A.off;
      j.ns = ig.ns;
      j.cs = ig.cs;
      j.wx = ig.wx;
      j.nimg = (int)ig.nimg;
      j.c = (int)ig.c;
      j.hp = (int)hp;
      j.wp = (int)wp;
      j.off_h = ig.off_h;
      j.ub_h = ig.ub_h;
      j.off_w = ig.off_w;
      j.ub_w = ig.ub_w;
      e.img = 1;
      e.img_slot = (int)ig.wo;
      e.img_rows = 128 / e.img_slot;
      e.img_wo = (int)ig.wo;
      e.img_ho = (int)ig.ho;
      e.img_hgroups = (int)((ig.ho + e.img_rows - 1) / e.img_rows);
      e.img_kh = (int)ig.kh;
      e.img_kw = (int)ig.kw;
      e.img_cblocks = (int)(ig.c / 64);
      e.img_a_mask = t.a_mask;
      e.tiles_m = (int)(ig.nimg * e.img_hgroups);
      if (t.nseg == 1) {
        t.halo = e;
        // halo tiles keep 512-element chunks: their first chunk drains while
        // the tile's last k blocks run (measured faster than one chunk)
        t.halo.chunk_blocks = 0;
        t.halo_ok = ltb_tc_halo_geometry(t.halo, (int)wp);
      }
      // B' in the image's K order: k' = (kh * KW + kw) * C + c
      std::vector<int64_t> kstride(kd.size());
      {
        int64_t st = 1;
        for (int q = (int)kd.size() - 1; q >= 0; --q) {
          kstride[q] = st;
          st *= d.size[kd[q]];
        }
      }
      auto pos = [&](int dim) { return (int)(std::find(kd.begin(), kd.end(), dim) - kd.begin()); };
      const int pc = pos(ig.c_dim), ph = pos(ig.kh_dim), pw = pos(ig.kw_dim);
      std::vector<int64_t> perm(con.K);
      for (int64_t kh = 0, k2 = 0; kh < ig.kh; ++kh)
        for (int64_t kw = 0; kw < ig.kw; ++kw)
          for (int64_t ch = 0; ch < ig.c; ++ch, ++k2)
            perm[k2] = ch * kstride[pc] + kh * kstride[ph] + kw * kstride[pw];
      std::vector<int64_t> bk(con.K);
      for (int64_t q = 0; q < con.K; ++q) bk[q] = ktab_b[perm[q]];
      ar.add(bk, &t.b_k);
      if (t.b_ng) {
        std::vector<int32_t> vk;
        for (int g = B.g0; g < B.g0 + B.ng; ++g) {
          auto gk = table(kd, d.guards[g].coef, 0);
          for (int64_t q = 0; q < con.K; ++q) vk.push_back((int32_t)gk[perm[q]]);
        }
        ar.add(vk, &t.bg_k);
      }
      auto rb = table(nd, B.coef, B.off);
      t.b_dense = B.ng == 0 && rb[0] == 0 && arith(rb, &t.b_ldr) && arith(bk, &t.b_ldk);
      t.b_kcontig = unit_frac(bk) >= unit_frac(rb);
    }
    // narrow outputs take 128-wide tiles (no half-empty MMA), the rest 256
    set_tile_n(t, con.N <= 128 ? 128 : 256, 0);
  }
}

// Per-device facts, queried once per process and device (compiles are
// frequent in a serving loop: every new size is a new loop tree).
struct DeviceInfo {
  bool ready = false;
  int sms = 0;
  int64_t bandwidth_gbs = 0;
};

const DeviceInfo& device_info(int dev) {
  static std::mutex mu;
  static std::map<int, DeviceInfo> info;
  std::lock_guard<std::mutex> g(mu);
  DeviceInfo& d = info[dev];
  if (d.ready) return d;
  CUDA_TRY(cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev));
  int memclk_khz = 0, bus_bits = 0;
  cudaDeviceGetAttribute(&memclk_khz, cudaDevAttrMemoryClockRate, dev);
  cudaDeviceGetAttribute(&bus_bits, cudaDevAttrGlobalMemoryBusWidth, dev);
  cudaGetLastError();
  d.bandwidth_gbs = (int64_t)(2.0 * memclk_khz * 1e3 * (bus_bits / 8) / 1e9);
  // host buffers are staged through the stream-ordered pool; keep what it
  // reserved across synchronisations instead of unmapping it every time
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  cudaGetLastError();
  d.ready = true;
  return d;
}

void pin_cfg(ltb_compiled* c, int i);

void compile_device(ltb_compiled* c) {
  CUDA_TRY(cudaGetDevice(&c->device));
  const DeviceInfo& di = device_info(c->device);
  c->sms = di.sms;
  c->bandwidth_gbs = di.bandwidth_gbs;
  auto& P = c->plan;
  const int ns = (int)P.stages.size();
  c->split_of.assign(ns, 1);
  c->gemm_of.assign(ns, -1);
  for (int i = 0; i < ns; ++i) {
    auto& st = P.stages[i];
    if (st.family == ltb::Family::reduce_split) {
      const int64_t outs = stage_outs(st.dev);
      int64_t splits = (4LL * c->sms + outs - 1) / outs;
      splits = std::min<int64_t>(splits, std::max<int64_t>(1, st.dev.red_total / 4096));
      // a "parallel" loop over the reduced var: that many threads in all,
      // 256 per partial
      if (st.pins.parallel_red > 256) splits = (st.pins.parallel_red + 255) / 256;
      splits = std::max<int64_t>(1, std::min<int64_t>(splits, 2048));
      c->split_of[i] = (int)splits;
      st.dev.split = (int)splits;
      st.dev.partial_buf = P.num_slots();
      P.scratch_elems.push_back(outs * splits);
    } else {
      st.dev.split = 1;
    }
  }
  Arena ar;
  c->gemms.reserve(ns);  // table pointers are patched in place: no realloc
  for (int i = 0; i < ns; ++i) {
    if (P.stages[i].family != ltb::Family::contraction) continue;
    c->gemm_of[i] = (int)c->gemms.size();
    c->gemms.emplace_back();
    GemmTables& t = c->gemms.back();
    t.stage = i;
    build_gemm(c, i, t, ar);
  }
  // scratch: one block, every slot 256-byte aligned
  c->scratch_off.clear();
  size_t off = 0;
  for (auto e : P.scratch_elems) {
    c->scratch_off.push_back(off);
    off += ((size_t)std::max<int64_t>(e, 1) * 4 + 255) / 256 * 256;
  }
  c->scratch_bytes = off;  // allocated on the first run without caller scratch
  std::vector<LtbStage> hs;
  for (auto& st : P.stages) hs.push_back(st.dev);
  ar.add(hs, &c->d_stages);
  ar.finalize(c->owned);
  int launches = 0;
  for (int i = 0; i < ns; ++i) {
    auto& st = P.stages[i];
    if (st.family == ltb::Family::row_chain) {
      if (st.rows_from == i) launches++;
    } else if (st.family == ltb::Family::contraction) {
      const auto& t = c->gemms[c->gemm_of[i]];
      // tensor cores: pack A, pack B, GEMM (image operands: one packing launch)
      launches += (int)t.nbatch * (t.tc ? (t.img ? 2 : 3) : 1);
    } else {
      launches += c->split_of[i] > 1 ? 2 : 1;
    }
  }
  c->launches = launches;
  c->cfg.assign(ns, LtbCfg{0, 0, 0});
  for (int i = 0; i < ns; ++i) {
    if (c->gemm_of[i] >= 0 && c->gemms[c->gemm_of[i]].tc)
      c->cfg[i].variant = c->gemms[c->gemm_of[i]].bn;
    pin_cfg(c, i);
  }
}

// How a run treats one caller buffer (ltb_run_plan reports it).  The
// kernels read and write a buffer in place only when it is device memory
// of the compiled object's device, or managed memory, and 16-byte aligned:
// the elementwise, window and softmax kernels move 16-byte vectors wherever
// a row's offsets allow, and the tensor-core operand packers and the TMA
// engine need 16-byte aligned addresses.  Every other buffer a run accepts
// is staged through an aligned device copy.
enum BufKind {
  kBufHost = 0,        // pageable or pinned host memory: staged
  kBufDevice = 1,      // device memory of this device, aligned: in place
  kBufManaged = 2,     // managed memory, aligned: in place (prefetched)
  kBufMisaligned = 3,  // device/managed memory off a 16-byte boundary: staged
  kBufForeign = -1,    // another GPU's memory: rejected (a peer access)
};

int buffer_kind(const void* p, int dev) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return kBufHost;
  }
  if (a.type == cudaMemoryTypeDevice && a.device != dev) return kBufForeign;
  if (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged) return kBufHost;
  if (reinterpret_cast<uintptr_t>(p) & 15) return kBufMisaligned;
  return a.type == cudaMemoryTypeManaged ? kBufManaged : kBufDevice;
}

const char* buffer_kind_text(int k) {
  switch (k) {
    case kBufHost: return "host memory: staged through device memory";
    case kBufDevice: return "device memory: read/written in place";
    case kBufManaged: return "managed memory: prefetched, read/written in place";
    case kBufMisaligned: return "device/managed memory off a 16-byte boundary: staged "
                                "through an aligned device copy";
    default: return "another device's memory: rejected";
  }
}

// Entry points that run kernels on caller buffers without staging
// (captured runs, batches, the autotuner) accept in-place buffers only.
void require_in_place(const void* p, int dev, const char* what) {
  if (!p) throw ltb::Error(std::string(what) + ": null buffer");
  const int k = buffer_kind(p, dev);
  if (k != kBufDevice && k != kBufManaged)
    throw ltb::Error(std::string(what) + " need 16-byte aligned device or managed buffers of the "
                     "compiled object's device; got " + buffer_kind_text(k));
}


// Launches of stage i (nothing for a row-chain member that is not the
// chain's first stage: the chain launches as one kernel).
cudaError_t launch_stage(ltb_compiled* c, int i, const LtbBufTable& bt, cudaStream_t st) {
  auto& P = c->plan;
  const int ns = (int)P.stages.size();
  const auto& s = P.stages[i];
  const LtbStage* d = c->d_stages + i;
  const LtbCfg& cfg = c->cfg[i];
  cudaError_t e = cudaSuccess;
  switch (s.family) {
    case ltb::Family::elementwise:
    case ltb::Family::reduce_serial:
      e = ltb_launch_nest(d, s.dev, bt, c->sms, st, cfg);
      break;
    case ltb::Family::reduce_parallel:
    case ltb::Family::reduce_split:
      e = ltb_launch_reduce(d, s.dev, bt, c->split_of[i], c->sms, st, cfg);
      break;
    case ltb::Family::row_chain: {
      if (s.rows_from != i) break;
      int n = 0;
      while (i + n < ns && P.stages[i + n].family == ltb::Family::row_chain &&
             P.stages[i + n].rows_from == i)
        n++;
      const LtbStage* hs[16];
      for (int k = 0; k < n && k < 16; ++k) hs[k] = &P.stages[i + k].dev;
      e = n <= 16 ? ltb_launch_row_chain(d, hs, n, bt, c->sms, st, cfg,
                                        timeout_flag(c->device, st))
                   : cudaErrorInvalidValue;
      break;
    }
    case ltb::Family::contraction: {
      const GemmTables& t = c->gemms[c->gemm_of[i]];
      for (int64_t b = 0; b < t.nbatch && e == cudaSuccess; ++b) {
        LtbGemmProblem p{};
        const LtbLoad& A = s.dev.loads[s.con.a_load];
        const LtbLoad& B = s.dev.loads[s.con.b_load];
        p.a = {bt.p[A.buf] + t.a_boff[b], t.a_row, t.a_k, t.a_dense ? 1 : 0, t.a_ldr, t.a_ldk,
               t.a_ng, t.ag_row, t.ag_k, t.ag_ub};
        p.b = {bt.p[B.buf] + t.b_boff[b], t.b_row, t.b_k, t.b_dense ? 1 : 0, t.b_ldr, t.b_ldk,
               t.b_ng, t.bg_row, t.bg_k, t.bg_ub};
        p.a.k32 = t.a_k32 ? 1 : 0;
        p.b.k32 = t.b_k32 ? 1 : 0;
        p.c = bt.p[s.dev.out_buf] + t.c_boff[b];
        p.crow = t.c_row;
        p.ccol = t.c_col;
        p.M = s.con.M;
        p.N = s.con.N;
        p.K = s.con.K;
        if (!t.tc) {
          e = ltb_launch_gemm_simt(p, c->sms, st, cfg.variant);
          continue;
        }
        void* ap = bt.p[t.a_slot];
        void* bp = bt.p[t.b_slot];
        alignas(64) unsigned char maps[640];  // A (hi image), B, A lo, A lo2, C
        if (t.img) {
          LtbImageJob j = image_job(t, p.a.base, ap);
          e = ltb_launch_pack_conv(j, p.b, p.N, p.K, bp, t.Kp, t.nseg, t.b_mask, t.b_kcontig,
                                   t.b_off32, st);
          // halo boxes: the tile's rows + kh - 1, full width
          if (e == cudaSuccess && halo_form(t.epi))
            e = ltb_make_tmap_image(maps, j.hi, j.nimg, j.hp, j.wp, j.c, t.halo.img_slot,
                                    t.halo.img_rows + t.halo.img_kh - 1);
          else if (e == cudaSuccess)
            e = ltb_make_tmap_image(maps, j.hi, j.nimg, j.hp, j.wp, j.c, t.prob.img_wo);
          if (e == cudaSuccess)
            e = ltb_make_tmap_image(maps + 256, j.lo ? j.lo : j.hi, j.nimg, j.hp, j.wp, j.c,
                                    t.prob.img_wo);
          if (e == cudaSuccess && j.lo2)
            e = ltb_make_tmap_image(maps + 384, j.lo2, j.nimg, j.hp, j.wp, j.c, t.prob.img_wo);
        } else {
          e = ltb_launch_pack(p.a, p.M, p.K, ap, t.Kp, t.nseg, t.a_mask, t.a_kcontig, t.a_off32,
                              c->sms, st);
          if (e == cudaSuccess) e = ltb_make_tmap(maps, ap, p.M, t.Kp, ltb_tc_tile_m());
        }
        if (e == cudaSuccess && !t.img)  // image operands packed B' with the image
          e = ltb_launch_pack(p.b, p.N, p.K, bp, t.Kp, t.nseg, t.b_mask, t.b_kcontig, t.b_off32,
                              c->sms, st);
        if (e == cudaSuccess) e = ltb_make_tmap(maps + 128, bp, p.N, t.Kp, b_box_rows(t));
        const bool c_tma = t.c_tma && !halo_form(t.epi) && aligned16(p.c + t.c_row0);
        if (e == cudaSuccess && c_tma)
          e = ltb_make_tmap_c(maps + 512, p.c + t.c_row0, p.M, p.N, t.c_ld);
        if (e == cudaSuccess) {
          LtbTcProblem one = halo_form(t.epi) ? t.halo : t.prob;
          one.c_tma = c_tma ? 1 : 0;
          one.group_m = t.prob.group_m;
          one.c = p.c;
          one.crow = t.c_row;
          one.ccol = t.c_col;
          e = ltb_launch_gemm_tc(variant_code(t), nullptr, 1, t.tiles, nullptr, c->sms,
                                 timeout_flag(c->device, st), st,
                                 &one, maps, maps + 128, t.img ? maps + 256 : nullptr,
                                 t.img_kinds == 3 ? maps + 384 : nullptr,
                                 c_tma ? maps + 512 : nullptr);
        }
      }
      break;
    }
  }
  return e;
}

void launch_plan(ltb_compiled* c, const LtbBufTable& bt, cudaStream_t st) {
  const int ns = (int)c->plan.stages.size();
  for (int i = 0; i < ns; ++i) {
    const cudaError_t e = launch_stage(c, i, bt, st);
    if (e != cudaSuccess)
      throw CudaFailure(std::string("launch of stage ") + std::to_string(i) + " (" +
                        c->plan.stages[i].text + "): " + cudaGetErrorString(e));
  }
}

// Apply a schedule to stage i (the tile width of a tensor-core contraction
// changes its tile count).
// The launch choices a stage's loop annotations pin (StagePins), on top of
// whatever schedule it has: "parallel" over output vars fixes threads x
// CTAs of the grid-stride families (and the CTA count of the per-output
// reduction), "parallel" over reduced vars the threads per output of the
// tree reduction (split-K counts are fixed when the object is compiled),
// "unroll" 4 (or 2) the work items per thread of the pooling window kernel.
void pin_cfg(ltb_compiled* c, int i) {
  const auto& s = c->plan.stages[i];
  const ltb::StagePins& pn = s.pins;
  if (!pn.any()) return;
  LtbCfg& cf = c->cfg[i];
  auto warp_round = [](int64_t t) {
    t = std::max<int64_t>(32, std::min<int64_t>(t, 256));
    return (int)(t / 32 * 32);
  };
  switch (s.family) {
    case ltb::Family::elementwise:
    case ltb::Family::reduce_serial:
      if (pn.parallel_out) {
        const int t = warp_round(pn.cta_threads ? pn.cta_threads : pn.parallel_out);
        cf.threads = t;
        cf.grid = (int)std::min<int64_t>((pn.parallel_out + t - 1) / t, 1 << 30);
      }
      if (pn.unroll) cf.variant = pn.unroll >= 4 ? 4 : 2;
      break;
    case ltb::Family::reduce_parallel:
    case ltb::Family::reduce_split:
      if (pn.parallel_red) cf.threads = warp_round(pn.parallel_red);
      if (pn.parallel_out) cf.grid = (int)std::min<int64_t>(pn.parallel_out, 1 << 30);
      break;
    default:
      break;
  }
}

void apply_cfg(ltb_compiled* c, int i, const LtbCfg& cfg) {
  c->cfg[i] = cfg;
  pin_cfg(c, i);
  const int g = c->gemm_of[i];
  if (g >= 0 && c->gemms[g].tc) {
    // variant: tile width | form, form 0: row-store (or TMA-store)
    // epilogue, 1: transposed epilogue, 2: two CTAs per SM (128 wide only),
    // 3: halo image tiles, 5: halo image tiles on CTA pairs (133); 258:
    // 256 x 256 tiles on CTA pairs
    const int v = cfg.variant;
    const int bn = v == 256 || v == 257 || v == 258 ? 256 : 128;
    const int epi = v == 129 || v == 257 ? 1
                    : v == 130              ? 2
                    : v == 131              ? 3
                    : v == 258              ? 4
                    : v == 133              ? 5
                                            : 0;
    set_tile_n(c->gemms[g], bn, epi);  // 131, 133 and 258 fall back where they do not apply
    c->cfg[i].variant = variant_code(c->gemms[g]);
    // cta_per_sm of a contraction: the raster group (row blocks swept together)
    c->gemms[g].prob.group_m = cfg.cta_per_sm;
  }
}

int run_impl(ltb_compiled* c, void* const* memory, int n, int sync,
             void* stream, void* scratch) {
  if (!c) return fail(LTB_ERR_INVALID, "null compiled object");
  auto& P = c->plan;
  if (n != P.n_in + P.n_out)
    return fail(LTB_ERR_INVALID, "expected " + std::to_string(P.n_in + P.n_out) +
                                     " buffers, got " + std::to_string(n));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  std::unique_lock<std::mutex> lock(c->mu, std::defer_lock);
  const bool default_scratch = !scratch;
  if (!scratch) {
    lock.lock();
    if (!c->scratch && c->scratch_bytes) {
      if (cudaMalloc(&c->scratch, c->scratch_bytes) != cudaSuccess) {
        cudaGetLastError();
        return fail(LTB_ERR_CUDA, "scratch allocation failed");
      }
      c->owned.push_back(c->scratch);
    }
    scratch = c->scratch;
  }
  LtbBufTable bt{};
  if (P.num_slots() > LTB_MAXBUF)
    return fail(LTB_ERR_UNSUPPORTED, "too many buffers for one launch table");
  std::vector<std::pair<int, void*>> staged;  // slot, host pointer
  std::vector<void*> temps;
  try {
    CUDA_TRY(cudaSetDevice(c->device));
    // every buffer in host memory and a plain linear map: stage the copies
    // chunk by chunk on two streams, so each chunk's download overlaps the
    // next chunk's upload (the host link runs both directions at once)
    // one pointer-attribute query per buffer per run
    int kind[LTB_MAXBUF];
    bool all_host = true;
    for (int i = 0; i < n; ++i) {
      if (!memory[i]) return fail(LTB_ERR_INVALID, "null buffer " + std::to_string(i));
      kind[i] = buffer_kind(memory[i], c->device);
      if (kind[i] == kBufForeign)
        return fail(LTB_ERR_INVALID, "buffer " + std::to_string(i) + ": " +
                                         buffer_kind_text(kind[i]));
      all_host = all_host && kind[i] == kBufHost;
    }
    if (scratch && (reinterpret_cast<uintptr_t>(scratch) & 255))
      return fail(LTB_ERR_INVALID, "caller scratch must be 256-byte aligned");
    constexpr int64_t kChunk = int64_t(1) << 23;  // elements per chunk (32 MB of FP32)
    const int64_t total = P.n_out ? P.io_elems[P.n_in] : 0;
    bool same = true;
    for (int i = 0; i < n; ++i) same = same && P.io_elems[i] == total;
    if (all_host && same && total >= 2 * kChunk && P.stages.size() == 1 &&
        P.stages[0].family == ltb::Family::elementwise && ltb_linear_range_ok(P.stages[0].dev)) {
      for (int i = 0; i < n; ++i) {
        void* d = nullptr;
        CUDA_TRY(cudaMallocAsync(&d, (size_t)total * 4, st));
        temps.push_back(d);
        bt.p[i] = static_cast<float*>(d);
      }
      cudaStream_t aux;
      {
        std::lock_guard<std::mutex> g(c->aux_mu);
        if (!c->aux) CUDA_TRY(cudaStreamCreateWithFlags(&c->aux, cudaStreamNonBlocking));
        aux = c->aux;
      }
      cudaEvent_t e0 = nullptr, e1 = nullptr;
      CUDA_TRY(cudaEventCreateWithFlags(&e0, cudaEventDisableTiming));
      CUDA_TRY(cudaEventCreateWithFlags(&e1, cudaEventDisableTiming));
      CUDA_TRY(cudaEventRecord(e0, st));
      CUDA_TRY(cudaStreamWaitEvent(aux, e0, 0));  // the allocations above are visible
      int k = 0;
      for (int64_t lo = 0; lo < total; lo += kChunk, ++k) {
        cudaStream_t s = (k & 1) ? aux : st;
        const int64_t cn = std::min<int64_t>(kChunk, total - lo);
        for (int i = 0; i < P.n_in; ++i)
          CUDA_TRY(cudaMemcpyAsync(bt.p[i] + lo, static_cast<const float*>(memory[i]) + lo,
                                   (size_t)cn * 4, cudaMemcpyHostToDevice, s));
        CUDA_TRY(ltb_launch_linear_range(P.stages[0].dev, bt, lo, cn, c->sms, s, c->cfg[0]));
        for (int j = P.n_in; j < n; ++j)
          CUDA_TRY(cudaMemcpyAsync(static_cast<float*>(memory[j]) + lo, bt.p[j] + lo,
                                   (size_t)cn * 4, cudaMemcpyDeviceToHost, s));
      }
      CUDA_TRY(cudaEventRecord(e1, aux));
      CUDA_TRY(cudaStreamWaitEvent(st, e1, 0));
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      for (void* d : temps) CUDA_TRY(cudaFreeAsync(d, st));
      if (sync) CUDA_TRY(cudaStreamSynchronize(st));
      return LTB_OK;
    }
    // managed buffers (the reference's "cuda" hardware allocates them) move
    // in bulk before the launch instead of page by page on first touch
    std::vector<int> managed;
    for (int i = 0; i < n; ++i)
      if (kind[i] == kBufManaged) {
        managed.push_back(i);
        const size_t bytes = (size_t)std::max<int64_t>(P.io_elems[i], 1) * 4;
        if (cudaMemPrefetchAsync(memory[i], bytes, c->device, st) != cudaSuccess)
          cudaGetLastError();  // advisory only
      }
    for (int i = 0; i < n; ++i) {
      if (kind[i] == kBufDevice || kind[i] == kBufManaged) {
        bt.p[i] = static_cast<float*>(memory[i]);
        continue;
      }
      // host memory, or device/managed memory off a 16-byte boundary:
      // an aligned device copy (cudaMallocAsync blocks are 256-byte aligned)
      const size_t bytes = (size_t)std::max<int64_t>(P.io_elems[i], 1) * 4;
      void* d = nullptr;
      CUDA_TRY(cudaMallocAsync(&d, bytes, st));
      temps.push_back(d);
      if (i < P.n_in)
        CUDA_TRY(cudaMemcpyAsync(d, memory[i], bytes, cudaMemcpyDefault, st));
      else
        staged.push_back({i, memory[i]});
      bt.p[i] = static_cast<float*>(d);
    }
    for (size_t k = 0; k < P.scratch_elems.size(); ++k)
      bt.p[P.n_in + P.n_out + k] =
          reinterpret_cast<float*>(static_cast<char*>(scratch) + c->scratch_off[k]);
    // The default scratch is shared by every run of this object that brings
    // none: this run's kernels wait (on the device) for the previous such
    // run, which may still be executing on another stream.  Skipped while
    // the stream is being captured (an event recorded outside a capture
    // cannot be waited on inside it).
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    CUDA_TRY(cudaStreamIsCapturing(st, &cap));
    const bool order = default_scratch && c->scratch_bytes && cap == cudaStreamCaptureStatusNone;
    if (order) {
      if (!c->scratch_done)
        CUDA_TRY(cudaEventCreateWithFlags(&c->scratch_done, cudaEventDisableTiming));
      else
        CUDA_TRY(cudaStreamWaitEvent(st, c->scratch_done, 0));
    }
    launch_plan(c, bt, st);
    if (order) CUDA_TRY(cudaEventRecord(c->scratch_done, st));
    for (auto& s : staged) {
      const size_t bytes = (size_t)std::max<int64_t>(P.io_elems[s.first], 1) * 4;
      CUDA_TRY(cudaMemcpyAsync(s.second, bt.p[s.first], bytes, cudaMemcpyDefault, st));
    }
    for (void* d : temps) CUDA_TRY(cudaFreeAsync(d, st));
    // a synchronous run's managed outputs go back to the host in bulk: the
    // caller waits for them in order to read them there
    if (sync)
      for (int i : managed)
        if (i >= P.n_in) {
          const size_t bytes = (size_t)std::max<int64_t>(P.io_elems[i], 1) * 4;
          if (cudaMemPrefetchAsync(memory[i], bytes, cudaCpuDeviceId, st) != cudaSuccess)
            cudaGetLastError();
        }
    // host outputs are written by stream-ordered copies: with sync == 0 they
    // are complete once the stream is (Compiled::async)
    if (sync) {
      CUDA_TRY(cudaStreamSynchronize(st));
      if (take_timeout(c->device, st))
        return fail(LTB_ERR_TIMEOUT, "a bounded wait in a kernel on this stream gave up");
    }
  } catch (const CudaFailure& e) {
    return fail(LTB_ERR_CUDA, e.what());
  } catch (const std::exception& e) {
    return fail(LTB_ERR_INVALID, e.what());
  }
  return LTB_OK;
}

int copy_out(const std::string& s, char* buf, size_t len) {
  if (!buf || !len) return fail(LTB_ERR_INVALID, "empty output buffer");
  size_t m = std::min(len - 1, s.size());
  memcpy(buf, s.data(), m);
  buf[m] = 0;
  return LTB_OK;
}

// ------------------------------------------------------------- schedules
// Autotuned launch schedules, cached per process by a hash of the IR text
// (which carries every size, so structure and shape together) and the
// compile options, and persisted as text that keeps the IR itself (a
// portable record: the serialized loop tree plus its schedule).
struct TuneEntry {
  std::string ir, opts;
  int sms = 0;
  std::vector<LtbCfg> cfg;
  std::vector<double> us;
};
std::mutex g_tune_mu;
std::map<uint64_t, TuneEntry> g_tune;

std::string canon_options(const ltb::LowerOptions& o) {
  return "precision=" + std::to_string((int)o.precision) + ";fuse_rows=" +
         std::to_string((int)o.fuse_rows) + ";tensor_cores=" +
         std::to_string((int)o.use_tensor_cores) + ";kahan_threshold=" +
         std::to_string(o.kahan_threshold);
}

uint64_t fnv1a(const std::string& a, const std::string& b) {
  uint64_t h = 1469598103934665603ULL;
  auto mix = [&](const std::string& x) {
    for (unsigned char ch : x) {
      h ^= ch;
      h *= 1099511628211ULL;
    }
    h ^= 0x1f;
    h *= 1099511628211ULL;
  };
  mix(a);
  mix(b);
  return h;
}

// The schedule in the vocabulary of LoopTree annotations.
std::string describe(ltb_compiled* c, int i) {
  const auto& s = c->plan.stages[i];
  const LtbCfg& f = c->cfg[i];
  std::ostringstream o;
  if (s.family == ltb::Family::contraction) {
    const auto& t = c->gemms[c->gemm_of[i]];
    if (t.tc)
      o << (t.epi == 4 ? "tile(256x256x64 on CTA pairs, cta_group::2)" : "tile(128x")
        << (t.epi == 4 ? "" : std::to_string(t.bn) + "x64)")
        << " tensor_cores(tcgen05) parallel(persistent, " << t.tiles << " tiles) raster("
        << (t.prob.group_m ? t.prob.group_m : 16) << " row blocks) epilogue("
        << (t.c_tma && t.epi != 2 && !halo_form(t.epi) ? "TMA stores where aligned, else " : "")
        << (t.epi == 1 ? "smem transpose" : t.epi == 2 ? "row stores, 2 CTAs/SM" : "row stores")
        << ")"
        << (t.epi == 5 ? " on CTA pairs (cta_group::2, M = 256, half the weights per CTA)" : "")
        << (halo_form(t.epi)
                ? " implicit_conv(halo tiles: one 4-D TMA box per tile and channel block, "
                  "every (kh, kw) shift read in place; weights resident in shared memory)"
            : t.img ? " implicit_conv(A from NHWC image via 4-D TMA)"
                    : "");
    else {
      LtbGemmProblem q{};
      q.M = s.con.M;
      q.N = s.con.N;
      const int tile = ltb_simt_tile(q, c->sms, f.variant);
      o << "tile(" << tile << "x" << tile << ") cuda_cores";
    }
    return o.str();
  }
  o << "parallel(grid=SMs x " << (f.cta_per_sm ? std::to_string(f.cta_per_sm) : "resident")
    << ") threaded(" << (f.threads ? std::to_string(f.threads) : "default") << ")";
  if (f.variant) o << " variant(" << f.variant << ")";
  return o.str();
}

std::vector<LtbCfg> candidates(ltb_compiled* c, int i) {
  auto& P = c->plan;
  const auto& s = P.stages[i];
  LtbCfg buf[128];
  int n = 0;
  switch (s.family) {
    case ltb::Family::elementwise:
    case ltb::Family::reduce_serial:
      n = ltb_nest_candidates(s.dev, buf, 128);
      break;
    case ltb::Family::reduce_parallel:
    case ltb::Family::reduce_split:
      n = ltb_reduce_candidates(s.dev, buf, 128);
      break;
    case ltb::Family::row_chain: {
      int m = 0;
      const LtbStage* hs[16];
      while (i + m < (int)P.stages.size() && m < 16 &&
             P.stages[i + m].family == ltb::Family::row_chain && P.stages[i + m].rows_from == i) {
        hs[m] = &P.stages[i + m].dev;
        m++;
      }
      n = ltb_row_chain_candidates(hs, m, buf, 128);
      break;
    }
    case ltb::Family::contraction:
      if (c->gemms[c->gemm_of[i]].tc) {
        for (int v : {128, 129, 130, 256, 257, 258})
          if (v != 258 || !c->gemms[c->gemm_of[i]].img)
            for (int gm : {0, 8, 32}) buf[n++] = LtbCfg{gm, 0, v};
        if (c->gemms[c->gemm_of[i]].halo_ok) {
          buf[n++] = LtbCfg{0, 0, 131};
          buf[n++] = LtbCfg{0, 0, 133};
        }
      } else {  // CUDA-core tiles
        buf[n++] = LtbCfg{0, 0, 64};
        buf[n++] = LtbCfg{0, 0, 128};
      }
      break;
  }
  return std::vector<LtbCfg>(buf, buf + n);
}

// Mean device time (microseconds) of stage i's launches over reps runs;
// infinity if a launch is rejected.
double time_stage(ltb_compiled* c, int i, const LtbBufTable& bt, cudaStream_t st, int reps,
                  cudaEvent_t e0, cudaEvent_t e1) {
  if (launch_stage(c, i, bt, st) != cudaSuccess) {
    cudaGetLastError();
    return std::numeric_limits<double>::infinity();
  }
  CUDA_TRY(cudaEventRecord(e0, st));
  for (int r = 0; r < reps; ++r)
    if (launch_stage(c, i, bt, st) != cudaSuccess) {
      cudaGetLastError();
      CUDA_TRY(cudaStreamSynchronize(st));
      return std::numeric_limits<double>::infinity();
    }
  CUDA_TRY(cudaEventRecord(e1, st));
  CUDA_TRY(cudaEventSynchronize(e1));
  float ms = 0.f;
  CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
  return 1e3 * ms / reps;
}

void record_schedule(ltb_compiled* c, const std::vector<double>& us) {
  TuneEntry e;
  e.ir = c->ir_text;
  e.opts = canon_options(c->opt);
  e.sms = c->sms;
  e.cfg = c->cfg;
  e.us = us;
  e.us.resize(e.cfg.size(), 0.0);
  std::lock_guard<std::mutex> g(g_tune_mu);
  g_tune[c->key] = std::move(e);
}

// ---------------------------------------------------- schedule as IR text
// The launch schedule of the grid-stride and tree-reduction stages written
// back into the loop tree as the reference's own vocabulary: the stage's
// outermost unsplit output loop v of size S becomes
//   v (S / (G*T), S % (G*T)), v (G) "parallel", v (T) "parallel"
// (G CTAs of T threads), and the innermost unsplit reduced loop r of size
// R of a tree reduction becomes r (R / T, R % T), r (T) "parallel" (T
// threads per output).  Splits keep every loop's visiting order, so values
// are unchanged (reductions still fold in ascending index order).  Stages
// whose choices the vocabulary cannot express (fused row kernels, tile
// kernels) keep their schedule in the schedule cache only.
std::vector<std::string> split_keep(const std::string& s, char sep) {
  std::vector<std::string> out;
  size_t a = 0;
  while (true) {
    size_t b = s.find(sep, a);
    out.push_back(s.substr(a, b == std::string::npos ? std::string::npos : b - a));
    if (b == std::string::npos) break;
    a = b + 1;
  }
  return out;
}

struct OrderEdit {
  std::vector<std::pair<int, ltb::LoopSize>> order;
  std::vector<std::string> annots;
};

OrderEdit node_order(const ltb::Node& N) {
  OrderEdit e;
  e.order = N.order;
  e.annots.assign(N.order.size(), "");
  for (size_t i = 0; i < N.order.size() && i < N.loop_annotations.size(); ++i)
    e.annots[i] = N.loop_annotations[i];
  return e;
}

// replace entry i by the given loops (same var), keeping annotations elsewhere
void split_entry(OrderEdit& e, size_t i, const std::vector<std::pair<ltb::LoopSize, std::string>>& parts) {
  const int v = e.order[i].first;
  std::vector<std::pair<int, ltb::LoopSize>> o(e.order.begin(), e.order.begin() + i);
  std::vector<std::string> a(e.annots.begin(), e.annots.begin() + i);
  for (auto& p : parts) {
    o.push_back({v, p.first});
    a.push_back(p.second);
  }
  o.insert(o.end(), e.order.begin() + i + 1, e.order.end());
  a.insert(a.end(), e.annots.begin() + i + 1, e.annots.end());
  e.order = o;
  e.annots = a;
}

// the unsplit entry of a var in `vars`: outermost (first) or innermost (last)
int unsplit_entry(const OrderEdit& e, const std::vector<int>& vars, bool innermost) {
  int found = -1;
  for (size_t i = 0; i < e.order.size(); ++i) {
    const int v = e.order[i].first;
    if (std::find(vars.begin(), vars.end(), v) == vars.end()) continue;
    int n = 0;
    for (auto& o : e.order) n += o.first == v;
    if (n != 1 || e.order[i].second.tail != 0) continue;
    if (!innermost) return (int)i;
    found = (int)i;
  }
  return found;
}

std::string schedule_ir(ltb_compiled* c) {
  auto lines = split_keep(c->ir_text, '\n');
  std::vector<size_t> node_line;
  for (size_t l = 0; l < lines.size(); ++l)
    if (lines[l].rfind("n:", 0) == 0) node_line.push_back(l);
  const auto& P = c->plan;
  std::map<int, OrderEdit> edits;
  for (size_t i = 0; i < P.stages.size(); ++i) {
    const auto& s = P.stages[i];
    const LtbCfg& cf = c->cfg[i];
    if (s.pins.any() || s.node < 0 || s.node >= (int)node_line.size()) continue;
    const bool grid_stride = s.family == ltb::Family::elementwise ||
                             s.family == ltb::Family::reduce_serial;
    const bool tree = s.family == ltb::Family::reduce_parallel;
    if (!grid_stride && !tree) continue;
    const ltb::Node& N = c->ir.nodes[s.node];
    OrderEdit e = edits.count(s.node) ? edits[s.node] : node_order(N);
    const int nout = s.dev.nout;
    std::vector<int> outv(s.dim_vars.begin(), s.dim_vars.begin() + nout);
    std::vector<int> redv(s.dim_vars.begin() + nout, s.dim_vars.end());
    const int T = cf.threads > 0 ? cf.threads
                                 : grid_stride ? 256 : (s.dev.red_total >= 256 ? 256 : 128);
    const int64_t G = cf.grid > 0 ? cf.grid : cf.cta_per_sm > 0 ? (int64_t)c->sms * cf.cta_per_sm : 0;
    if (tree) {
      const int k = unsplit_entry(e, redv, true);
      if (k >= 0 && e.order[k].second.size >= T) {
        const int64_t R = e.order[k].second.size;
        split_entry(e, (size_t)k, {{{R / T, R % T}, e.annots[k]}, {{T, 0}, "parallel"}});
      }
    }
    if (G > 0) {
      const int k = unsplit_entry(e, outv, false);
      const int64_t GT = G * (grid_stride ? T : 1);
      if (k >= 0 && e.order[k].second.size >= GT) {
        const int64_t S = e.order[k].second.size;
        if (grid_stride)
          split_entry(e, (size_t)k, {{{S / GT, S % GT}, e.annots[k]}, {{G, 0}, "parallel"},
                                     {{T, 0}, "parallel"}});
        else
          split_entry(e, (size_t)k, {{{S / G, S % G}, e.annots[k]}, {{G, 0}, "parallel"}});
      }
    }
    edits[s.node] = e;
  }
  for (auto& kv : edits) {
    auto f = split_keep(lines[node_line[kv.first]], ':');
    if (f.size() != 11) continue;
    std::ostringstream o, a;
    for (auto& x : kv.second.order) o << x.first << ";" << x.second.size << ";" << x.second.tail << ",";
    for (auto& x : kv.second.annots) a << x << ",";
    const std::string old_order = f[7];
    f[7] = o.str();
    f[9] = a.str();
    std::string ln;
    for (size_t j = 0; j < f.size(); ++j) ln += (j ? ":" : "") + f[j];
    lines[node_line[kv.first]] = ln;
    // a write fused into this node shares its loops in the reference's tree
    for (int w : c->ir.outputs) {
      const auto& W = c->ir.nodes[w];
      if (W.inputs.size() != 1 || W.inputs[0] != kv.first || edits.count(w)) continue;
      auto fw = split_keep(lines[node_line[w]], ':');
      if (fw.size() != 11 || fw[7] != old_order) continue;
      fw[7] = f[7];
      fw[9] = f[9];
      std::string lw;
      for (size_t j = 0; j < fw.size(); ++j) lw += (j ? ":" : "") + fw[j];
      lines[node_line[w]] = lw;
    }
  }
  std::string out;
  for (size_t l = 0; l < lines.size(); ++l) out += (l ? "\n" : "") + lines[l];
  return out;
}

// Schedules from the cache, if this IR + options were tuned before.
void lookup_schedule(ltb_compiled* c) {
  c->key = fnv1a(c->ir_text, canon_options(c->opt));
  std::lock_guard<std::mutex> g(g_tune_mu);
  auto it = g_tune.find(c->key);
  if (it == g_tune.end()) return;
  const TuneEntry& e = it->second;
  if (e.ir != c->ir_text || e.sms != c->sms || e.cfg.size() != c->cfg.size()) return;
  for (size_t i = 0; i < e.cfg.size(); ++i) apply_cfg(c, (int)i, e.cfg[i]);
  c->tuned = true;
}

}  // namespace

// ------------------------------------------------------------------ batch
// Many compiled contractions (e.g. 512 uneven matmuls) run as one grouped
// launch: one pack launch over every operand, one persistent tensor-core
// launch over every tile of every problem (or one grouped FP32 launch),
// optionally captured once into a CUDA graph and replayed.
struct ltb_batch {
  int device = 0, sms = 148;
  bool tc = false;
  int n = 0;
  LtbPackJob* d_jobs = nullptr;
  int njobs = 0;
  int64_t pack_tiles = 0;
  int pack_chunk = 0, pack_cta_per_sm = 0;  // grouped pack schedule (0: defaults)
  bool pack_dense = false;  // every pack job of a dense mode (the faster kernel)
  bool pack_one_seg = false;  // every pack job with one segment (plain BF16)
  std::vector<LtbImageJob> img_jobs;        // image operands, repacked before the pack
  // tensor-core problems grouped by schedule variant (kGroupCode), one
  // persistent launch per non-empty group
  LtbTcProblem* d_tc[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  int ntc[6] = {0, 0, 0, 0, 0, 0};
  int64_t tc_tiles[6] = {0, 0, 0, 0, 0, 0};
  int tc_tma[6] = {0, 0, 0, 0, 0, 0};  // a problem of the group has a TMA-stored output
  // each group's tiles dealt longest first to the least-loaded work unit of
  // its persistent launch (tile_order): unit u runs order[ostart[u] ..
  // ostart[u + 1])
  int* d_order[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  int* d_ostart[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  LtbGemmProblem* d_simt = nullptr;
  int64_t* d_simt_start = nullptr;
  int64_t simt_tiles = 0;
  int simt_modes = 0;  // tile loader forms every FP32 member allows
  int* d_err = nullptr;
  double flops = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<void*> owned;
};

namespace {

constexpr int kGroups = 6;
constexpr int kGroupCode[kGroups] = {128, 129, 256, 257, 130, 258};  // launch variant per group

int group_of(const GemmTables& t) {
  const int v = variant_code(t);
  for (int g = 0; g < kGroups; ++g)
    if (kGroupCode[g] == v) return g;
  return 0;
}

// A tile's cost for the assignment: its k blocks plus a fixed share for
// the drain and epilogue (about 4 k blocks of MMA time, measured on the
// batch's small-K tiles).
constexpr int64_t kTileFixedCost = 4;

// Longest-processing-time assignment of a group's tiles (problems in tile
// order, each with tiles_m x tiles_n tiles of ceil(Kp / 64) k blocks) to
// `units` work units: tiles by descending cost (stable, so a problem's
// tiles keep their raster order and run side by side), each to the unit
// with the least work so far.  Returns the per-unit tile lists
// concatenated and their start offsets.  Round-robin dealing leaves the
// slowest unit of the 512-matmul batch ~10% above the mean in a model of
// these costs; this leaves it at the mean.
void tile_order(const std::vector<LtbTcProblem>& probs, int64_t units, std::vector<int>* order,
                std::vector<int>* ostart) {
  std::vector<int64_t> cost;
  for (const auto& q : probs) {
    const int64_t n = (int64_t)q.tiles_m * q.tiles_n, kb = (q.Kp + 63) / 64;
    cost.insert(cost.end(), (size_t)n, kb + kTileFixedCost);
  }
  std::vector<int> idx(cost.size());
  for (size_t i = 0; i < idx.size(); ++i) idx[i] = (int)i;
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return cost[a] > cost[b]; });
  using Load = std::pair<int64_t, int64_t>;  // (work so far, unit)
  std::priority_queue<Load, std::vector<Load>, std::greater<Load>> heap;
  for (int64_t u = 0; u < units; ++u) heap.push({0, u});
  std::vector<std::vector<int>> lists((size_t)units);
  for (int t : idx) {
    Load l = heap.top();
    heap.pop();
    lists[(size_t)l.second].push_back(t);
    heap.push({l.first + cost[t], l.second});
  }
  order->clear();
  ostart->assign(1, 0);
  for (const auto& l : lists) {
    order->insert(order->end(), l.begin(), l.end());
    ostart->push_back((int)order->size());
  }
}

void batch_gemms(ltb_batch* b, cudaStream_t st) {
  for (int g = 0; g < kGroups; ++g)
    if (b->ntc[g])
      CUDA_TRY(ltb_launch_gemm_tc(kGroupCode[g], b->d_tc[g], b->ntc[g], b->tc_tiles[g], nullptr,
                                  b->sms, b->d_err, st, nullptr, nullptr, nullptr, nullptr,
                                  nullptr, nullptr, b->tc_tma[g], b->d_order[g],
                                  b->d_ostart[g]));
}

void batch_launch(ltb_batch* b, cudaStream_t st) {
  if (b->tc) {
    for (const auto& j : b->img_jobs) CUDA_TRY(ltb_launch_pack_image(j, st));
    CUDA_TRY(ltb_launch_pack_grouped(b->d_jobs, b->njobs, b->pack_tiles, b->sms, st, b->pack_chunk,
                                     b->pack_cta_per_sm, b->pack_dense, b->pack_one_seg));
    batch_gemms(b, st);
  } else {
    CUDA_TRY(ltb_launch_gemm_simt_grouped(b->d_simt, b->d_simt_start, b->n, b->simt_tiles,
                                           b->simt_modes, st));
  }
}

int batch_finish(ltb_batch* b, int sync, cudaStream_t st) {
  if (!sync) return LTB_OK;
  CUDA_TRY(cudaStreamSynchronize(st));
  int flag = 0;
  CUDA_TRY(cudaMemcpy(&flag, b->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (flag) {
    CUDA_TRY(cudaMemset(b->d_err, 0, sizeof(int)));
    return fail(LTB_ERR_TIMEOUT, "a bounded wait in a tensor-core kernel gave up");
  }
  return LTB_OK;
}

}  // namespace

extern "C" {

int ltb_abi_version(void) { return 1; }

int ltb_batch_create(ltb_compiled* const* cs, void* const* const* memories, int n,
                     ltb_batch** out) {
  if (!cs || !memories || n <= 0 || !out) return fail(LTB_ERR_INVALID, "bad batch arguments");
  *out = nullptr;
  auto b = new ltb_batch();
  try {
    b->n = n;
    b->device = cs[0]->device;
    b->sms = cs[0]->sms;
    // the batch's tables live on (and its launch shapes are asked of) the
    // members' device, whatever device is current
    CUDA_TRY(cudaSetDevice(b->device));
    std::vector<LtbPackJob> jobs;
    std::vector<LtbTcProblem> tcp[kGroups];
    std::vector<unsigned char> maps[kGroups];  // five 128-byte CUtensorMaps per problem
    std::vector<LtbGemmProblem> sp;
    std::vector<int64_t> sstart;
    for (int i = 0; i < n; ++i) {
      ltb_compiled* c = cs[i];
      if (!c || c->device != b->device)
        throw ltb::Error("batch members must be compiled on one device");
      if (c->plan.stages.size() != 1 || c->plan.stages[0].family != ltb::Family::contraction)
        throw ltb::Error("batch member " + std::to_string(i) + " is not a single contraction");
      const auto& s = c->plan.stages[0];
      const GemmTables& t = c->gemms[c->gemm_of[0]];
      if (t.nbatch != 1) throw ltb::Error("batched contractions cannot join a batch");
      if (i == 0) b->tc = t.tc;
      if (t.tc != b->tc || (t.tc && t.nseg != cs[0]->gemms[0].nseg))
        throw ltb::Error("batch members must share one precision");
      const int nio = c->plan.n_in + c->plan.n_out;
      if (!memories[i]) throw ltb::Error("batch member without buffers");
      for (int k = 0; k < nio; ++k) require_in_place(memories[i][k], b->device, "batches");
      auto ptr = [&](int slot) { return static_cast<float*>(memories[i][slot]); };
      const LtbLoad& A = s.dev.loads[s.con.a_load];
      const LtbLoad& B = s.dev.loads[s.con.b_load];
      LtbGemmProblem p{};
      p.a = {ptr(A.buf), t.a_row, t.a_k, t.a_dense ? 1 : 0, t.a_ldr, t.a_ldk, t.a_ng, t.ag_row,
             t.ag_k, t.ag_ub};
      p.b = {ptr(B.buf), t.b_row, t.b_k, t.b_dense ? 1 : 0, t.b_ldr, t.b_ldk, t.b_ng, t.bg_row,
             t.bg_k, t.bg_ub};
      p.a.k32 = t.a_k32 ? 1 : 0;
      p.b.k32 = t.b_k32 ? 1 : 0;
      p.c = ptr(s.dev.out_buf);
      p.crow = t.c_row;
      p.ccol = t.c_col;
      p.M = s.con.M;
      p.N = s.con.N;
      p.K = s.con.K;
      b->flops += 2.0 * p.M * p.N * p.K;
      if (b->tc) {
        auto job = [&](const LtbGemmOperand& op, int64_t rows, void* dst, int mask, bool kc,
                       bool off32) {
          LtbPackJob j{};
          j.op = op;
          j.out = dst;
          j.rows = rows;
          j.K = p.K;
          j.Kp = t.Kp;
          j.tiles_k = (int)((p.K + 63) / 64);
          j.tile_start = b->pack_tiles;
          j.nseg = t.nseg;
          j.seg_mask = mask;
          j.mode = ltb_pack_mode(op, rows, p.K, kc ? 1 : 0);
          j.off32 = off32 ? 1 : 0;
          b->pack_tiles += ltb_pack_tiles(rows, p.K);
          jobs.push_back(j);
        };
        void *ap = nullptr, *bp = nullptr;
        const size_t a_bytes =
            t.img ? (size_t)t.img_kinds * t.img_elems * 2 : (size_t)p.M * t.Kp * 2;
        CUDA_TRY(cudaMalloc(&ap, a_bytes));
        b->owned.push_back(ap);
        CUDA_TRY(cudaMalloc(&bp, (size_t)p.N * t.Kp * 2));
        b->owned.push_back(bp);
        if (!t.img) job(p.a, p.M, ap, t.a_mask, t.a_kcontig, t.a_off32);
        job(p.b, p.N, bp, t.b_mask, t.b_kcontig, t.b_off32);
        const int grp = group_of(t);
        auto& mv = maps[grp];
        mv.resize(mv.size() + 640);  // A (hi image), B, A lo image, A lo2 image, C
        unsigned char* m = mv.data() + mv.size() - 640;
        if (t.img) {
          const LtbImageJob j = image_job(t, p.a.base, ap);
          b->img_jobs.push_back(j);
          CUDA_TRY(ltb_make_tmap_image(m, j.hi, j.nimg, j.hp, j.wp, j.c, t.prob.img_wo));
          CUDA_TRY(ltb_make_tmap_image(m + 256, j.lo ? j.lo : j.hi, j.nimg, j.hp, j.wp, j.c,
                                       t.prob.img_wo));
          CUDA_TRY(ltb_make_tmap_image(m + 384, j.lo2 ? j.lo2 : j.lo ? j.lo : j.hi, j.nimg, j.hp,
                                       j.wp, j.c, t.prob.img_wo));
        } else {
          CUDA_TRY(ltb_make_tmap(m, ap, p.M, t.Kp, ltb_tc_tile_m()));
        }
        // (a halo-form member runs the per-row tiles of its width here)
        CUDA_TRY(
            ltb_make_tmap(m + 128, bp, p.N, t.Kp, halo_form(t.epi) ? t.bn : b_box_rows(t)));
        LtbTcProblem q = t.prob;
        q.c_tma = t.c_tma && aligned16(p.c + t.c_row0) ? 1 : 0;
        if (q.c_tma) CUDA_TRY(ltb_make_tmap_c(m + 512, p.c + t.c_row0, p.M, p.N, t.c_ld));
        b->tc_tma[grp] |= q.c_tma;
        q.c = p.c;
        q.crow = t.c_row;
        q.ccol = t.c_col;
        q.tile_start = b->tc_tiles[grp];
        // halo tiles are a single-launch form: in a group the member runs
        // its per-row image tiles at the same width
        b->tc_tiles[grp] += halo_form(t.epi) ? (int64_t)t.prob.tiles_m * t.prob.tiles_n : t.tiles;
        tcp[grp].push_back(q);
      } else {
        if (p.K > kSimtMaxK) throw ltb::Error("contraction too long for the FP32 kernel");
        sstart.push_back(b->simt_tiles);
        b->simt_tiles += ((p.M + 127) / 128) * ((p.N + 127) / 128);
        sp.push_back(p);
      }
    }
    b->njobs = (int)jobs.size();
    if (b->tc) {
      b->pack_dense = b->pack_one_seg = true;
      for (const auto& j : jobs) {
        b->pack_dense = b->pack_dense && (j.mode == kPackDenseK || j.mode == kPackDenseR);
        b->pack_one_seg = b->pack_one_seg && j.nseg == 1;
      }
      b->d_jobs = upload(jobs, b->owned);
      for (int g = 0; g < kGroups; ++g) {
        // tensor maps in device memory (cudaMalloc is 256-byte aligned)
        unsigned char* d_maps = upload(maps[g], b->owned);
        for (size_t i = 0; i < tcp[g].size(); ++i) {
          tcp[g][i].map_a = d_maps + 640 * i;
          tcp[g][i].map_b = d_maps + 640 * i + 128;
          tcp[g][i].map_a2 = d_maps + 640 * i + 256;
          tcp[g][i].map_a3 = d_maps + 640 * i + 384;
          tcp[g][i].map_c = d_maps + 640 * i + 512;
        }
        b->ntc[g] = (int)tcp[g].size();
        b->d_tc[g] = upload(tcp[g], b->owned);
        const int64_t units = ltb_tc_units(kGroupCode[g], b->tc_tiles[g], b->sms);
        if (b->ntc[g] && units > 0) {
          std::vector<int> order, ostart;
          tile_order(tcp[g], units, &order, &ostart);
          b->d_order[g] = upload(order, b->owned);
          b->d_ostart[g] = upload(ostart, b->owned);
        }
      }
    } else {
      b->d_simt = upload(sp, b->owned);
      b->d_simt_start = upload(sstart, b->owned);
      // one loader form per operand for the whole launch: the members' common
      // form, else the gather form, which serves every operand
      int am = -1, bm = -1;
      for (const auto& q : sp) {
        const int a = ltb_simt_mode(q.a, q.M, q.K, true), bb = ltb_simt_mode(q.b, q.N, q.K, false);
        am = am < 0 || am == a ? a : kSimtGather;
        bm = bm < 0 || bm == bb ? bb : kSimtGather;
      }
      b->simt_modes = std::max(am, 0) | std::max(bm, 0) << 4;
    }
    CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(&b->d_err), sizeof(int)));
    b->owned.push_back(b->d_err);
    CUDA_TRY(cudaMemset(b->d_err, 0, sizeof(int)));
  } catch (const CudaFailure& e) {
    for (void* p : b->owned) cudaFree(p);
    delete b;
    return fail(LTB_ERR_CUDA, e.what());
  } catch (const std::exception& e) {
    for (void* p : b->owned) cudaFree(p);
    delete b;
    return fail(LTB_ERR_INVALID, e.what());
  }
  *out = b;
  return LTB_OK;
}

int ltb_batch_run(ltb_batch* b, int sync, void* stream) {
  if (!b) return fail(LTB_ERR_INVALID, "null batch");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  try {
    CUDA_TRY(cudaSetDevice(b->device));
    if (b->exec)
      CUDA_TRY(cudaGraphLaunch(b->exec, st));
    else
      batch_launch(b, st);
    return batch_finish(b, sync, st);
  } catch (const std::exception& e) {
    return fail(LTB_ERR_CUDA, e.what());
  }
}

int ltb_batch_capture(ltb_batch* b, void* stream) {
  if (!b) return fail(LTB_ERR_INVALID, "null batch");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (!st) return fail(LTB_ERR_INVALID, "capture needs a non-default stream");
  try {
    CUDA_TRY(cudaSetDevice(b->device));
    if (b->exec) {
      cudaGraphExecDestroy(b->exec);
      cudaGraphDestroy(b->graph);
      b->exec = nullptr;
      b->graph = nullptr;
    }
    CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    try {
      batch_launch(b, st);
    } catch (...) {
      cudaGraph_t g;
      cudaStreamEndCapture(st, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    CUDA_TRY(cudaStreamEndCapture(st, &b->graph));
    CUDA_TRY(cudaGraphInstantiate(&b->exec, b->graph, 0));
  } catch (const std::exception& e) {
    return fail(LTB_ERR_CUDA, e.what());
  }
  return LTB_OK;
}

int ltb_batch_run_timed(ltb_batch* b, void* stream, float* pack_ms, float* gemm_ms) {
  if (!b || !pack_ms || !gemm_ms) return fail(LTB_ERR_INVALID, "null argument");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaEvent_t e0 = nullptr, e1 = nullptr, e2 = nullptr;
  try {
    CUDA_TRY(cudaSetDevice(b->device));
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    CUDA_TRY(cudaEventCreate(&e2));
    CUDA_TRY(cudaEventRecord(e0, st));
    for (const auto& j : b->img_jobs) CUDA_TRY(ltb_launch_pack_image(j, st));
    if (b->tc)
      CUDA_TRY(ltb_launch_pack_grouped(b->d_jobs, b->njobs, b->pack_tiles, b->sms, st,
                                       b->pack_chunk, b->pack_cta_per_sm, b->pack_dense,
                                       b->pack_one_seg));
    CUDA_TRY(cudaEventRecord(e1, st));
    if (b->tc)
      batch_gemms(b, st);
    else
      CUDA_TRY(ltb_launch_gemm_simt_grouped(b->d_simt, b->d_simt_start, b->n, b->simt_tiles,
                                           b->simt_modes, st));
    CUDA_TRY(cudaEventRecord(e2, st));
    CUDA_TRY(cudaEventSynchronize(e2));
    CUDA_TRY(cudaEventElapsedTime(pack_ms, e0, e1));
    CUDA_TRY(cudaEventElapsedTime(gemm_ms, e1, e2));
  } catch (const std::exception& e) {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (e2) cudaEventDestroy(e2);
    return fail(LTB_ERR_CUDA, e.what());
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaEventDestroy(e2);
  return batch_finish(b, 1, st);
}

int ltb_batch_set_schedule(ltb_batch* b, int pack_chunk, int pack_cta_per_sm) {
  if (!b || pack_chunk < 0 || pack_chunk > 4096 || pack_cta_per_sm < 0 || pack_cta_per_sm > 64)
    return fail(LTB_ERR_INVALID, "bad batch schedule");
  b->pack_chunk = pack_chunk;
  b->pack_cta_per_sm = pack_cta_per_sm;
  if (b->exec) {  // the captured graph holds the old launch shape
    cudaGraphExecDestroy(b->exec);
    cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
  }
  return LTB_OK;
}

int ltb_batch_int_property(ltb_batch* b, const char* name, int64_t* value) {
  if (!b || !name || !value) return fail(LTB_ERR_INVALID, "null argument");
  std::string k = name;
  if (k == "problems") *value = b->n;
  else if (k == "flops") *value = (int64_t)b->flops;
  else if (k == "launches") {  // image repacks, the grouped pack, one per non-empty group
    int64_t n = b->tc ? 1 + (int64_t)b->img_jobs.size() : 1;
    if (b->tc)
      for (int g = 0; g < kGroups; ++g) n += b->ntc[g] > 0;
    *value = n;
  } else if (k == "tiles") {
    int64_t n = b->tc ? 0 : b->simt_tiles;
    if (b->tc)
      for (int g = 0; g < kGroups; ++g) n += b->tc_tiles[g];
    *value = n;
  } else if (k == "tiles_128") *value = b->tc_tiles[0] + b->tc_tiles[1] + b->tc_tiles[4];
  else if (k == "tiles_256") *value = b->tc_tiles[2] + b->tc_tiles[3];
  else if (k == "tiles_pair") *value = b->tc_tiles[5];  // 256 x 256 tiles on CTA pairs
  else if (k == "graph") *value = b->exec ? 1 : 0;
  else if (k == "pack_chunk") *value = b->pack_chunk ? b->pack_chunk : 4;
  else if (k == "pack_cta_per_sm")
    *value = b->pack_cta_per_sm  ? b->pack_cta_per_sm
             : b->pack_dense && b->pack_one_seg ? 6
                                                 : 4;
  else return fail(LTB_ERR_INVALID, "unknown property " + k);
  return LTB_OK;
}

int ltb_batch_release(ltb_batch* b) {
  if (!b) return LTB_OK;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (void* p : b->owned) cudaFree(p);
  delete b;
  return LTB_OK;
}

const char* ltb_last_error(void) { return g_err.c_str(); }

int ltb_device_count(void) {
  // the set of visible devices is fixed for the life of the process
  static const int count = [] {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
      cudaGetLastError();
      return 0;
    }
    int ok = 0;
    for (int i = 0; i < n; ++i) {
      int major = 0;
      if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, i) == cudaSuccess &&
          major == 10)
        ok++;
    }
    cudaGetLastError();
    return ok;
  }();
  return count;
}

int ltb_plan(const char* ir_text, const char* options, char* buf, size_t len) {
  if (!ir_text) return fail(LTB_ERR_INVALID, "null IR text");
  try {
    auto opt = parse_options(options);
    auto g = ltb::parse_ir(ir_text);
    auto p = ltb::lower(g, opt);
    return copy_out(p.dump, buf, len);
  } catch (const ltb::Error& e) {
    return fail(LTB_ERR_UNSUPPORTED, e.what());
  } catch (const std::exception& e) {
    return fail(LTB_ERR_INVALID, e.what());
  }
}

int ltb_compile(const char* ir_text, const char* options, ltb_compiled** out) {
  if (!ir_text || !out) return fail(LTB_ERR_INVALID, "null argument");
  *out = nullptr;
  auto c = new ltb_compiled();
  try {
    c->ir_text = ir_text;
    c->opt = parse_options(options);
    c->ir = ltb::parse_ir(c->ir_text);
    c->plan = ltb::lower(c->ir, c->opt);
  } catch (const std::exception& e) {
    delete c;
    return fail(LTB_ERR_UNSUPPORTED, e.what());
  }
  if (ltb_device_count() == 0) {
    delete c;
    return fail(LTB_ERR_NO_DEVICE, "no sm_100 CUDA device visible");
  }
  try {
    ensure_flag_table(c->device);
    compile_device(c);
    lookup_schedule(c);
  } catch (const std::exception& e) {
    for (void* p : c->owned) cudaFree(p);
    delete c;
    return fail(LTB_ERR_CUDA, e.what());
  }
  *out = c;
  return LTB_OK;
}

int ltb_run(ltb_compiled* c, void* const* memory, int n, int sync, void* stream) {
  return run_impl(c, memory, n, sync, stream, nullptr);
}

int ltb_run_with_scratch(ltb_compiled* c, void* const* memory, int n, int sync,
                         void* stream, void* scratch) {
  if (c && c->scratch_bytes && !scratch)
    return fail(LTB_ERR_INVALID, "scratch pointer required");
  return run_impl(c, memory, n, sync, stream, scratch);
}

int ltb_schedule_ir(ltb_compiled* c, char* buf, size_t len) {
  if (!c) return fail(LTB_ERR_INVALID, "null compiled object");
  try {
    return copy_out(schedule_ir(c), buf, len);
  } catch (const std::exception& e) {
    return fail(LTB_ERR_INVALID, e.what());
  }
}

int ltb_run_plan(ltb_compiled* c, void* const* memory, int n, char* buf, size_t len) {
  if (!c || !memory) return fail(LTB_ERR_INVALID, "null argument");
  const auto& P = c->plan;
  if (n != P.n_in + P.n_out)
    return fail(LTB_ERR_INVALID, "expected " + std::to_string(P.n_in + P.n_out) +
                                     " buffers, got " + std::to_string(n));
  std::ostringstream ss;
  for (int i = 0; i < n; ++i) {
    if (!memory[i]) return fail(LTB_ERR_INVALID, "null buffer " + std::to_string(i));
    ss << (i < P.n_in ? "input " : "output ") << (i < P.n_in ? i : i - P.n_in) << ": "
       << buffer_kind_text(buffer_kind(memory[i], c->device)) << "\n";
  }
  return copy_out(ss.str(), buf, len);
}

int ltb_release(ltb_compiled* c) {
  if (!c) return LTB_OK;
  if (c->aux) cudaStreamDestroy(c->aux);
  if (c->scratch_done) cudaEventDestroy(c->scratch_done);
  for (void* p : c->owned) cudaFree(p);
  delete c;
  return LTB_OK;
}

int ltb_dump(ltb_compiled* c, char* buf, size_t len) {
  if (!c) return fail(LTB_ERR_INVALID, "null compiled object");
  return copy_out(c->plan.dump, buf, len);
}

int ltb_int_property(ltb_compiled* c, const char* name, int64_t* value) {
  if (!c || !name || !value) return fail(LTB_ERR_INVALID, "null argument");
  std::string k = name;
  if (k == "bandwidth") *value = c->bandwidth_gbs;
  else if (k == "stages") *value = (int64_t)c->plan.stages.size();
  else if (k == "launches") *value = c->launches;
  else if (k == "scratch_bytes") *value = (int64_t)c->scratch_bytes;
  else if (k == "inputs") *value = c->plan.n_in;
  else if (k == "outputs") *value = c->plan.n_out;
  else if (k == "algorithmic_bytes") *value = c->plan.algorithmic_bytes;
  else if (k == "flops") *value = (int64_t)c->plan.flops;
  else if (k == "tuned") *value = c->tuned ? 1 : 0;
  else if (k == "implicit_conv") {
    int64_t n = 0;
    for (const auto& t : c->gemms) n += t.img ? 1 : 0;
    *value = n;
  }
  else if (k == "tma_store_output") {  // tensor-core contractions whose C TMA can store
    int64_t n = 0;
    for (const auto& t : c->gemms) n += t.tc && t.c_tma ? 1 : 0;
    *value = n;
  }
  else return fail(LTB_ERR_INVALID, "unknown property " + k);
  return LTB_OK;
}

int ltb_io_sizes(ltb_compiled* c, int* n_in, int* n_out, int64_t* elems, int cap) {
  if (!c) return fail(LTB_ERR_INVALID, "null compiled object");
  if (n_in) *n_in = c->plan.n_in;
  if (n_out) *n_out = c->plan.n_out;
  for (int i = 0; elems && i < cap && i < (int)c->plan.io_elems.size(); ++i)
    elems[i] = c->plan.io_elems[i];
  return LTB_OK;
}

int ltb_alloc(size_t bytes, int managed, void** out) {
  if (!out) return fail(LTB_ERR_INVALID, "null output pointer");
  if (managed < 0 || managed > 2) return fail(LTB_ERR_INVALID, "bad allocation kind");
  cudaError_t e = managed == 1   ? cudaMallocManaged(out, bytes, cudaMemAttachGlobal)
                  : managed == 2 ? cudaHostAlloc(out, bytes, cudaHostAllocPortable)
                                 : cudaMalloc(out, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(LTB_ERR_CUDA, std::string("allocation failed: ") + cudaGetErrorString(e));
  }
  return LTB_OK;
}

int ltb_free(void* ptr) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, ptr) == cudaSuccess && a.type == cudaMemoryTypeHost) {
    const cudaError_t e = cudaFreeHost(ptr);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(LTB_ERR_CUDA, cudaGetErrorString(e));
    }
    return LTB_OK;
  }
  cudaGetLastError();
  cudaError_t e = cudaFree(ptr);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(LTB_ERR_CUDA, cudaGetErrorString(e));
  }
  return LTB_OK;
}

// ------------------------------------------------------- captured runs
struct ltb_graph {
  ltb_compiled* c = nullptr;
  int* flag = nullptr;  // timeout flag of the capture stream
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

int ltb_graph_create(ltb_compiled* c, void* const* memory, int n, void* scratch, void* stream,
                     ltb_graph** out) {
  if (!c || !memory || !out) return fail(LTB_ERR_INVALID, "null argument");
  *out = nullptr;
  auto& P = c->plan;
  if (n != P.n_in + P.n_out)
    return fail(LTB_ERR_INVALID, "expected " + std::to_string(P.n_in + P.n_out) +
                                     " buffers, got " + std::to_string(n));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaStream_t own = nullptr;
  auto g = new ltb_graph();
  g->c = c;
  try {
    CUDA_TRY(cudaSetDevice(c->device));
    LtbBufTable bt{};
    for (int i = 0; i < n; ++i) {
      require_in_place(memory[i], c->device, "captured runs");
      bt.p[i] = static_cast<float*>(memory[i]);
    }
    if (!scratch) {
      std::lock_guard<std::mutex> lock(c->mu);
      if (!c->scratch && c->scratch_bytes) {
        CUDA_TRY(cudaMalloc(&c->scratch, c->scratch_bytes));
        c->owned.push_back(c->scratch);
      }
      scratch = c->scratch;
    }
    for (size_t k = 0; k < P.scratch_elems.size(); ++k)
      bt.p[P.n_in + P.n_out + k] =
          reinterpret_cast<float*>(static_cast<char*>(scratch) + c->scratch_off[k]);
    if (!st) {  // the legacy default stream cannot be captured
      CUDA_TRY(cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking));
      st = own;
    }
    g->flag = timeout_flag(c->device, st);
    CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    try {
      launch_plan(c, bt, st);
    } catch (...) {
      cudaGraph_t tmp = nullptr;
      cudaStreamEndCapture(st, &tmp);
      if (tmp) cudaGraphDestroy(tmp);
      throw;
    }
    CUDA_TRY(cudaStreamEndCapture(st, &g->graph));
    CUDA_TRY(cudaGraphInstantiate(&g->exec, g->graph, 0));
  } catch (const CudaFailure& e) {
    if (own) cudaStreamDestroy(own);
    ltb_graph_release(g);
    return fail(LTB_ERR_CUDA, e.what());
  } catch (const std::exception& e) {
    if (own) cudaStreamDestroy(own);
    ltb_graph_release(g);
    return fail(LTB_ERR_INVALID, e.what());
  }
  if (own) cudaStreamDestroy(own);
  *out = g;
  return LTB_OK;
}

int ltb_graph_run(ltb_graph* g, int sync, void* stream) {
  if (!g || !g->exec) return fail(LTB_ERR_INVALID, "null captured run");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  try {
    CUDA_TRY(cudaSetDevice(g->c->device));
    CUDA_TRY(cudaGraphLaunch(g->exec, st));
    if (sync) {
      CUDA_TRY(cudaStreamSynchronize(st));
      // the graph's kernels raise the flag of the stream it was captured on
      int flag = 0;
      CUDA_TRY(cudaMemcpy(&flag, g->flag, sizeof(int), cudaMemcpyDeviceToHost));
      if (flag) {
        CUDA_TRY(cudaMemset(g->flag, 0, sizeof(int)));
        return fail(LTB_ERR_TIMEOUT, "a bounded wait in a kernel of this captured run gave up");
      }
    }
  } catch (const std::exception& e) {
    return fail(LTB_ERR_CUDA, e.what());
  }
  return LTB_OK;
}

int ltb_graph_release(ltb_graph* g) {
  if (!g) return LTB_OK;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  delete g;
  return LTB_OK;
}

// ------------------------------------------------------------ autotuner
int ltb_tune(ltb_compiled* c, void* const* memory, int n, void* stream, int reps, char* report,
             size_t len) {
  if (!c || !memory) return fail(LTB_ERR_INVALID, "null argument");
  auto& P = c->plan;
  if (n != P.n_in + P.n_out)
    return fail(LTB_ERR_INVALID, "expected " + std::to_string(P.n_in + P.n_out) +
                                     " buffers, got " + std::to_string(n));
  if (reps < 1) reps = 1;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  std::ostringstream rep;
  try {
    CUDA_TRY(cudaSetDevice(c->device));
    LtbBufTable bt{};
    for (int i = 0; i < n; ++i) {
      try {
        require_in_place(memory[i], c->device, "tuning runs");
      } catch (const std::exception& e) {
        return fail(LTB_ERR_INVALID, e.what());
      }
      bt.p[i] = static_cast<float*>(memory[i]);
    }
    {
      std::lock_guard<std::mutex> lock(c->mu);
      if (!c->scratch && c->scratch_bytes) {
        CUDA_TRY(cudaMalloc(&c->scratch, c->scratch_bytes));
        c->owned.push_back(c->scratch);
      }
    }
    for (size_t k = 0; k < P.scratch_elems.size(); ++k)
      bt.p[P.n_in + P.n_out + k] =
          reinterpret_cast<float*>(static_cast<char*>(c->scratch) + c->scratch_off[k]);
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    launch_plan(c, bt, st);  // every stage's inputs in place
    CUDA_TRY(cudaStreamSynchronize(st));
    std::vector<double> best_us(P.stages.size(), 0.0);
    for (int i = 0; i < (int)P.stages.size(); ++i) {
      const auto& s = P.stages[i];
      if (s.family == ltb::Family::row_chain && s.rows_from != i) continue;
      auto cands = candidates(c, i);
      const LtbCfg start = c->cfg[i];
      const double t0 = time_stage(c, i, bt, st, reps, e0, e1);
      LtbCfg best = start;
      double bt_us = t0;
      for (const auto& cand : cands) {
        apply_cfg(c, i, cand);
        const double t = time_stage(c, i, bt, st, reps, e0, e1);
        if (t < bt_us) {
          bt_us = t;
          best = c->cfg[i];
        }
      }
      apply_cfg(c, i, best);
      best_us[i] = bt_us;
      rep << "stage " << i << " " << s.text << "\n  " << describe(c, i) << "  "
          << std::fixed << std::setprecision(2) << bt_us << " us (default " << t0 << " us, "
          << cands.size() << " candidates)\n";
    }
    launch_plan(c, bt, st);  // outputs from the chosen schedules
    CUDA_TRY(cudaStreamSynchronize(st));
    if (take_timeout(c->device, st))
      throw ltb::Error("a bounded wait in a kernel gave up while tuning");
    c->tuned = true;
    record_schedule(c, best_us);
  } catch (const CudaFailure& e) {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    return fail(LTB_ERR_CUDA, e.what());
  } catch (const std::exception& e) {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    return fail(LTB_ERR_INVALID, e.what());
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (report && len) return copy_out(rep.str(), report, len);
  return LTB_OK;
}

int ltb_set_schedule(ltb_compiled* c, int stage, int cta_per_sm, int threads, int variant) {
  if (!c || stage < 0 || stage >= (int)c->cfg.size())
    return fail(LTB_ERR_INVALID, "bad compiled object or stage index");
  if (cta_per_sm < 0 || cta_per_sm > 1024 || !(threads == 0 || threads == 64 ||
                                                threads == 128 || threads == 256 ||
                                                threads == 512))
    return fail(LTB_ERR_INVALID, "bad schedule");
  apply_cfg(c, stage, LtbCfg{cta_per_sm, threads, variant});
  return LTB_OK;
}

int ltb_get_schedule(ltb_compiled* c, int stage, int* cta_per_sm, int* threads, int* variant) {
  if (!c || stage < 0 || stage >= (int)c->cfg.size())
    return fail(LTB_ERR_INVALID, "bad compiled object or stage index");
  if (cta_per_sm) *cta_per_sm = c->cfg[stage].cta_per_sm;
  if (threads) *threads = c->cfg[stage].threads;
  if (variant) *variant = c->cfg[stage].variant;
  return LTB_OK;
}

int ltb_tune_record(ltb_compiled* c) {
  if (!c) return fail(LTB_ERR_INVALID, "null compiled object");
  record_schedule(c, {});
  c->tuned = true;
  return LTB_OK;
}

int64_t ltb_tune_entries(void) {
  std::lock_guard<std::mutex> g(g_tune_mu);
  return (int64_t)g_tune.size();
}

int ltb_tune_clear(void) {
  std::lock_guard<std::mutex> g(g_tune_mu);
  g_tune.clear();
  return LTB_OK;
}

// Text file: a header line, then per entry
//   entry <sms> <stages> <ir bytes> <options bytes>\n<ir><options>\n
//   <cta_per_sm> <threads> <variant> <us>\n   (one line per stage)
int ltb_tune_save(const char* path) {
  if (!path) return fail(LTB_ERR_INVALID, "null path");
  std::ofstream f(path, std::ios::binary | std::ios::trunc);
  if (!f) return fail(LTB_ERR_INVALID, std::string("cannot write ") + path);
  std::lock_guard<std::mutex> g(g_tune_mu);
  f << "loop_tool_b200 schedules 1\n";
  for (const auto& kv : g_tune) {
    const TuneEntry& e = kv.second;
    f << "entry " << e.sms << " " << e.cfg.size() << " " << e.ir.size() << " " << e.opts.size()
      << "\n";
    f.write(e.ir.data(), (std::streamsize)e.ir.size());
    f.write(e.opts.data(), (std::streamsize)e.opts.size());
    f << "\n";
    for (size_t i = 0; i < e.cfg.size(); ++i)
      f << e.cfg[i].cta_per_sm << " " << e.cfg[i].threads << " " << e.cfg[i].variant << " "
        << (i < e.us.size() ? e.us[i] : 0.0) << "\n";
  }
  return f ? LTB_OK : fail(LTB_ERR_INVALID, std::string("write failed: ") + path);
}

int ltb_tune_load(const char* path) {
  if (!path) return fail(LTB_ERR_INVALID, "null path");
  std::ifstream f(path, std::ios::binary);
  if (!f) return fail(LTB_ERR_INVALID, std::string("cannot read ") + path);
  std::string line;
  if (!std::getline(f, line) || line != "loop_tool_b200 schedules 1")
    return fail(LTB_ERR_INVALID, "not a schedule file");
  std::vector<TuneEntry> got;
  while (std::getline(f, line)) {
    if (line.empty()) continue;
    std::istringstream h(line);
    std::string tag;
    size_t ns = 0, irb = 0, ob = 0;
    TuneEntry e;
    if (!(h >> tag >> e.sms >> ns >> irb >> ob) || tag != "entry" || ns > 4096 ||
        irb > (64u << 20) || ob > 4096)
      return fail(LTB_ERR_INVALID, "malformed schedule entry");
    e.ir.resize(irb);
    e.opts.resize(ob);
    if (irb) f.read(&e.ir[0], (std::streamsize)irb);
    if (ob) f.read(&e.opts[0], (std::streamsize)ob);
    std::getline(f, line);
    if (!f) return fail(LTB_ERR_INVALID, "truncated schedule entry");
    for (size_t i = 0; i < ns; ++i) {
      LtbCfg cfg{};
      double us = 0;
      if (!std::getline(f, line)) return fail(LTB_ERR_INVALID, "truncated schedule entry");
      std::istringstream r(line);
      if (!(r >> cfg.cta_per_sm >> cfg.threads >> cfg.variant >> us))
        return fail(LTB_ERR_INVALID, "malformed schedule line");
      e.cfg.push_back(cfg);
      e.us.push_back(us);
    }
    got.push_back(std::move(e));
  }
  std::lock_guard<std::mutex> g(g_tune_mu);
  for (auto& e : got) {
    const uint64_t k = fnv1a(e.ir, e.opts);
    g_tune[k] = std::move(e);
  }
  return LTB_OK;
}

int ltb_check_bounded_wait(int64_t limit_cycles, void* stream, int* completed, int* drained) {
  if (limit_cycles < 1 || limit_cycles > 4000000000LL)
    return fail(LTB_ERR_INVALID, "limit_cycles must be in [1, 4e9]");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  try {
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(LTB_ERR_INVALID, "device index out of range");
    ensure_flag_table(dev);
    int status[2] = {-1, -1};
    CUDA_TRY(ltb_launch_wait_check(timeout_flag(dev, st), limit_cycles, status, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    if (completed) *completed = status[0];
    if (drained) *drained = status[1];
    if (take_timeout(dev, st))
      return fail(LTB_ERR_TIMEOUT, "the bounded wait gave up (the self-check's expected outcome)");
  } catch (const std::exception& e) {
    return fail(LTB_ERR_CUDA, e.what());
  }
  return LTB_OK;
}

int ltb_synchronize(void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail(LTB_ERR_CUDA, cudaGetErrorString(e));
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return LTB_OK;
  }
  try {
    if (take_timeout(dev, st))
      return fail(LTB_ERR_TIMEOUT, "a bounded wait in a kernel on this stream gave up");
  } catch (const std::exception& ex) {
    return fail(LTB_ERR_CUDA, ex.what());
  }
  return LTB_OK;
}

}  // extern "C"
