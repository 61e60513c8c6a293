// Native continuous-batching request loop over the C ABI (declared in
// include/loop_tool_b200.h, "serving").  Host code only: it compiles loop
// trees with ltb_compile, runs them with ltb_run_with_scratch on per-slot
// streams and workspaces, and generates request inputs on the device
// (serve_fill.cu).  The reference has no serving loop: its lazy frontend
// runs one program at a time, synchronously (lazy.h:249-258).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/loop_tool_b200.h"
#include "kernels.h"

cudaError_t ltb_launch_fill_block(float* x, int64_t rows, int64_t cols, int64_t true_rows,
                                  int64_t true_cols, uint64_t seed, float scale, int sms,
                                  cudaStream_t st);

namespace {

constexpr size_t kAlign = 256;  // bytes between the regions of a workspace

size_t up(size_t b) { return (b + kAlign - 1) / kAlign * kAlign; }

// A compiled loop tree and the layout of a request's regions in a slot
// workspace: inputs, outputs, then run scratch.
struct Program {
  ltb_compiled* c = nullptr;
  int n_in = 0, n_out = 0;
  std::vector<int64_t> elems;
  std::vector<size_t> off;  // byte offset of each I/O buffer
  size_t scratch_off = 0, scratch_bytes = 0, ws_bytes = 0;
  int64_t request_bytes = 0;  // I/O + scratch (the budget's unit)
};

int err(int code, const std::string& m) { return ltb_set_last_error(code, m.c_str()); }

}  // namespace

struct ltb_server {
  int device = 0, sms = 148, slots = 0;
  int64_t budget = 0;
  std::string options;
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> events;
  std::vector<void*> ws;
  std::vector<size_t> ws_bytes;
  std::unordered_map<std::string, Program> programs;
  int64_t compiles = 0;
  double compile_s = 0.0;
};

namespace {

// The request's compiled program (compiling it on first use).
int program_of(ltb_server* s, const ltb_request& r, Program** out) {
  if (!r.ir_text) return err(LTB_ERR_INVALID, "request without a loop tree");
  auto it = s->programs.find(r.ir_text);
  if (it == s->programs.end()) {
    const auto t0 = std::chrono::steady_clock::now();
    Program p;
    int rc = ltb_compile(r.ir_text, s->options.c_str(), &p.c);
    if (rc != LTB_OK) return rc;
    int64_t elems[LTB_SERVE_MAX_IO];
    rc = ltb_io_sizes(p.c, &p.n_in, &p.n_out, elems, LTB_SERVE_MAX_IO);
    if (rc == LTB_OK && p.n_in + p.n_out > LTB_SERVE_MAX_IO)
      rc = err(LTB_ERR_UNSUPPORTED, "loop tree with more than LTB_SERVE_MAX_IO buffers");
    int64_t sb = 0;
    if (rc == LTB_OK) rc = ltb_int_property(p.c, "scratch_bytes", &sb);
    if (rc != LTB_OK) {
      ltb_release(p.c);
      return rc;
    }
    size_t o = 0;
    for (int i = 0; i < p.n_in + p.n_out; ++i) {
      p.elems.push_back(elems[i]);
      p.off.push_back(o);
      o += up((size_t)std::max<int64_t>(elems[i], 1) * 4);
      p.request_bytes += elems[i] * 4;
    }
    p.scratch_off = o;
    p.scratch_bytes = (size_t)sb;
    p.ws_bytes = o + up(p.scratch_bytes);
    p.request_bytes += sb;
    s->compile_s +=
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    s->compiles++;
    it = s->programs.emplace(r.ir_text, std::move(p)).first;
  }
  *out = &it->second;
  return LTB_OK;
}

int check_request(const Program& p, const ltb_request& r, int idx) {
  if (r.n_io != p.n_in + p.n_out)
    return err(LTB_ERR_INVALID, "request " + std::to_string(idx) + ": " + std::to_string(r.n_io) +
                                    " buffer descriptions for a loop tree of " +
                                    std::to_string(p.n_in + p.n_out) + " buffers");
  for (int i = 0; i < r.n_io; ++i) {
    const ltb_block& b = r.io[i];
    if (b.rows * b.cols != p.elems[i] || b.true_rows > b.rows || b.true_cols > b.cols ||
        b.true_rows < 0 || b.true_cols < 0)
      return err(LTB_ERR_INVALID, "request " + std::to_string(idx) + ": buffer " +
                                      std::to_string(i) + " does not match the loop tree");
  }
  return LTB_OK;
}

// Grows slot k's workspace to at least `bytes` (stream-ordered: the slot is
// idle, its previous work ordered before the free on its own stream).
int grow(ltb_server* s, int k, size_t bytes) {
  if (s->ws_bytes[k] >= bytes) return LTB_OK;
  cudaStream_t st = s->streams[k];
  if (s->ws[k] && cudaFreeAsync(s->ws[k], st) != cudaSuccess)
    return err(LTB_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
  s->ws[k] = nullptr;
  s->ws_bytes[k] = 0;
  if (cudaMallocAsync(&s->ws[k], bytes, st) != cudaSuccess) {
    cudaGetLastError();
    return err(LTB_ERR_CUDA, "slot workspace allocation failed");
  }
  s->ws_bytes[k] = bytes;
  return LTB_OK;
}

int launch(ltb_server* s, const ltb_request& r, Program& p, int k) {
  int rc = grow(s, k, p.ws_bytes);
  if (rc != LTB_OK) return rc;
  cudaStream_t st = s->streams[k];
  char* base = static_cast<char*>(s->ws[k]);
  void* mem[LTB_SERVE_MAX_IO];
  for (int i = 0; i < p.n_in + p.n_out; ++i) {
    mem[i] = base + p.off[i];
    if (i < p.n_in) {
      const ltb_block& b = r.io[i];
      if (ltb_launch_fill_block(static_cast<float*>(mem[i]), b.rows, b.cols, b.true_rows,
                                b.true_cols, r.seed * 1000003ull + (uint64_t)i,
                                b.scale != 0.f ? b.scale : 1.f, s->sms, st) != cudaSuccess)
        return err(LTB_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
    }
  }
  rc = ltb_run_with_scratch(p.c, mem, p.n_in + p.n_out, 0, st,
                            p.scratch_bytes ? base + p.scratch_off : nullptr);
  if (rc != LTB_OK) return rc;
  if (r.host_out && p.n_out > 0) {
    const ltb_block& b = r.io[p.n_in];
    if (cudaMemcpy2DAsync(r.host_out, (size_t)b.true_cols * 4, mem[p.n_in], (size_t)b.cols * 4,
                          (size_t)b.true_cols * 4, (size_t)b.true_rows, cudaMemcpyDeviceToHost,
                          st) != cudaSuccess)
      return err(LTB_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
  }
  if (cudaEventRecord(s->events[k], st) != cudaSuccess)
    return err(LTB_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
  return LTB_OK;
}

double pct(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const double pos = q * (double)(v.size() - 1);
  const size_t i = (size_t)pos;
  const double f = pos - (double)i;
  return i + 1 < v.size() ? v[i] * (1 - f) + v[i + 1] * f : v[i];
}

}  // namespace

extern "C" {

int ltb_server_create(int slots, int64_t hbm_budget, const char* options, ltb_server** out) {
  if (!out || slots < 1 || slots > 1024 || hbm_budget <= 0)
    return err(LTB_ERR_INVALID, "bad server arguments");
  *out = nullptr;
  auto s = new ltb_server();
  s->slots = slots;
  s->budget = hbm_budget;
  s->options = options ? options : "";
  if (cudaGetDevice(&s->device) != cudaSuccess ||
      cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, s->device) !=
          cudaSuccess) {
    cudaGetLastError();
    delete s;
    return err(LTB_ERR_NO_DEVICE, "no CUDA device");
  }
  for (int k = 0; k < slots; ++k) {
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      if (st) cudaStreamDestroy(st);
      ltb_server_release(s);
      return err(LTB_ERR_CUDA, "stream / event creation failed");
    }
    s->streams.push_back(st);
    s->events.push_back(ev);
    s->ws.push_back(nullptr);
    s->ws_bytes.push_back(0);
  }
  *out = s;
  return LTB_OK;
}

int ltb_server_prepare(ltb_server* s, const ltb_request* reqs, int n, int64_t* reserved) {
  if (!s || (!reqs && n > 0)) return err(LTB_ERR_INVALID, "null argument");
  size_t need = 0;
  for (int i = 0; i < n; ++i) {
    Program* p = nullptr;
    int rc = program_of(s, reqs[i], &p);
    if (rc == LTB_OK) rc = check_request(*p, reqs[i], i);
    if (rc != LTB_OK) return rc;
    need = std::max(need, p->ws_bytes);
  }
  const size_t per_slot = std::min<size_t>(need, (size_t)(s->budget / s->slots));
  for (int k = 0; k < s->slots; ++k) {
    const int rc = grow(s, k, per_slot);
    if (rc != LTB_OK) return rc;
  }
  size_t held = 0;
  for (int k = 0; k < s->slots; ++k) {
    if (cudaStreamSynchronize(s->streams[k]) != cudaSuccess)
      return err(LTB_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
    held += s->ws_bytes[k];
  }
  if (reserved) *reserved = (int64_t)held;
  return LTB_OK;
}

int ltb_server_serve(ltb_server* s, const ltb_request* reqs, int n, double time_scale,
                     ltb_serve_stats* stats, double* latency_s) {
  using clock = std::chrono::steady_clock;
  if (!s || (!reqs && n > 0)) return err(LTB_ERR_INVALID, "null argument");
  if (cudaSetDevice(s->device) != cudaSuccess)
    return err(LTB_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
  // every request checked (and compiled) before the clock starts
  std::vector<Program*> prog(n, nullptr);
  for (int i = 0; i < n; ++i) {
    int rc = program_of(s, reqs[i], &prog[i]);
    if (rc == LTB_OK) rc = check_request(*prog[i], reqs[i], i);
    if (rc == LTB_OK && prog[i]->request_bytes > s->budget)
      rc = err(LTB_ERR_INVALID, "request " + std::to_string(i) + " needs " +
                                    std::to_string(prog[i]->request_bytes) +
                                    " bytes, more than the budget");
    if (rc != LTB_OK) return rc;
  }
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return reqs[a].arrival_s < reqs[b].arrival_s; });
  std::vector<double> done(n, -1.0);
  std::vector<int> inflight(s->slots, -1);
  std::vector<int> free_slots;
  for (int k = s->slots - 1; k >= 0; --k) free_slots.push_back(k);
  std::deque<int> pending;
  int64_t used = 0, peak_used = 0, peak_inflight = 0, live = 0;
  size_t next = 0;
  const auto t0 = clock::now();
  auto now_s = [&] { return std::chrono::duration<double>(clock::now() - t0).count(); };
  while (next < order.size() || !pending.empty() || live > 0) {
    const double now = now_s();
    while (next < order.size() && reqs[order[next]].arrival_s * time_scale <= now)
      pending.push_back(order[next++]);
    for (int k = 0; k < s->slots; ++k) {
      const int r = inflight[k];
      if (r < 0) continue;
      const cudaError_t q = cudaEventQuery(s->events[k]);
      if (q == cudaErrorNotReady) continue;
      if (q != cudaSuccess) return err(LTB_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
      done[r] = now_s();
      used -= prog[r]->request_bytes;
      inflight[k] = -1;
      free_slots.push_back(k);
      --live;
    }
    while (!pending.empty() && !free_slots.empty() &&
           used + prog[pending.front()]->request_bytes <= s->budget) {
      const int r = pending.front();
      pending.pop_front();
      const int k = free_slots.back();
      free_slots.pop_back();
      const int rc = launch(s, reqs[r], *prog[r], k);
      if (rc != LTB_OK) return rc;
      used += prog[r]->request_bytes;
      inflight[k] = r;
      ++live;
      peak_used = std::max(peak_used, used);
      peak_inflight = std::max(peak_inflight, live);
    }
    if (pending.empty() && live == 0 && next < order.size()) {
      const double wait = reqs[order[next]].arrival_s * time_scale - now_s();
      if (wait > 0)
        std::this_thread::sleep_for(std::chrono::duration<double>(std::min(wait, 0.001)));
    }
  }
  for (int k = 0; k < s->slots; ++k)
    if (cudaStreamSynchronize(s->streams[k]) != cudaSuccess)
      return err(LTB_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
  std::vector<double> lat(n);
  double first = 1e300, last = 0.0, sum = 0.0;
  for (int i = 0; i < n; ++i) {
    lat[i] = done[i] - reqs[i].arrival_s * time_scale;
    first = std::min(first, reqs[i].arrival_s * time_scale);
    last = std::max(last, done[i]);
    sum += lat[i];
    if (latency_s) latency_s[i] = lat[i];
  }
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->requests = n;
    stats->compiles = s->compiles;
    stats->compile_s = s->compile_s;
    stats->peak_inflight = peak_inflight;
    stats->peak_bytes = peak_used;
    stats->span_s = n ? last - first : 0.0;
    stats->req_per_s = stats->span_s > 0 ? n / stats->span_s : 0.0;
    stats->p50_ms = 1e3 * pct(lat, 0.50);
    stats->p99_ms = 1e3 * pct(lat, 0.99);
    stats->mean_ms = n ? 1e3 * sum / n : 0.0;
  }
  return LTB_OK;
}

int ltb_server_release(ltb_server* s) {
  if (!s) return LTB_OK;
  for (size_t k = 0; k < s->streams.size(); ++k) {
    if (s->streams[k]) cudaStreamSynchronize(s->streams[k]);
    if (s->ws[k]) cudaFreeAsync(s->ws[k], s->streams[k]);
  }
  for (size_t k = 0; k < s->streams.size(); ++k) {
    if (s->streams[k]) {
      cudaStreamSynchronize(s->streams[k]);
      cudaStreamDestroy(s->streams[k]);
    }
    if (s->events[k]) cudaEventDestroy(s->events[k]);
  }
  for (auto& kv : s->programs) ltb_release(kv.second.c);
  delete s;
  return LTB_OK;
}

}  // extern "C"
