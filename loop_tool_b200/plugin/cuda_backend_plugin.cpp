// loop_tool plugin: registers the B200 backend as the "cuda" Backend and
// Hardware of a loop_tool build.  This is the reference-side binding: it is
// compiled against loop_tool's own headers (include/loop_tool/backend.h,
// hardware.h, serialization.h) and forwards to the C ABI in
// include/loop_tool_b200.h.  Load it like any backend plugin:
//   loop_tool::loadLibrary("libloop_tool_cuda_b200.so")   (backend.cpp:63-65)
//   lt.load_lib("libloop_tool_cuda_b200.so")              (python.cpp:87)
// Registration happens only when an sm_100 device is visible, as the
// reference's static registration does (src/backends/cuda/cuda.cpp:1030-1041).
#include <loop_tool/backend.h>
#include <loop_tool/hardware.h>
#include <loop_tool/serialization.h>

#include <cstdlib>
#include <memory>
#include <string>
#include <vector>

#include "loop_tool_b200.h"

namespace {

const char* options() {
  // e.g. LOOP_TOOL_B200_OPTIONS="precision=bf16x3"
  const char* o = std::getenv("LOOP_TOOL_B200_OPTIONS");
  return o ? o : "";
}

// Schedule cache file (LOOP_TOOL_B200_SCHEDULES): loaded at registration so
// compiles of loop trees tuned before start from their tuned schedules; with
// LOOP_TOOL_B200_AUTOTUNE=1 the first run of every new loop tree is tuned
// (on its own buffers) and the file rewritten.
const char* schedule_file() { return std::getenv("LOOP_TOOL_B200_SCHEDULES"); }
bool autotune() {
  const char* a = std::getenv("LOOP_TOOL_B200_AUTOTUNE");
  return a && std::string(a) == "1";
}

// LOOP_TOOL_B200_HOST_MEMORY=pinned: the "cuda" hardware hands out pinned
// host memory instead of managed memory (both CPU and GPU compatible).
int alloc_kind() {
  const char* m = std::getenv("LOOP_TOOL_B200_HOST_MEMORY");
  return m && std::string(m) == "pinned" ? 2 : 1;
}

// CudaGPUHardware (cuda.cpp:800-816): managed memory, usable by the CPU too.
struct B200Hardware : public loop_tool::Hardware {
  B200Hardware() : Hardware("cuda", ltb_device_count()) {}
  loop_tool::Memory alloc(size_t size) override {
    void* p = nullptr;
    ASSERT(ltb_alloc(size, alloc_kind(), &p) == LTB_OK) << ltb_last_error();
    return loop_tool::Memory{0x1 | (1 << id_), p};
  }
  void free(loop_tool::Memory& m) override {
    ltb_free(m.address);
    m.address = nullptr;
    m.compatible = 0;
  }
};

// CudaCompiled (cuda.cpp:818-851, 893-971): the LoopTree crosses the ABI as
// its serialized IR (serialization.cpp:175-237).
struct B200Compiled : public loop_tool::Compiled {
  ltb_compiled* h = nullptr;
  explicit B200Compiled(const loop_tool::LoopTree& lt) {
    const std::string text = loop_tool::serialize(lt.ir);
    ASSERT(ltb_compile(text.c_str(), options(), &h) == LTB_OK) << ltb_last_error();
    int64_t bw = 0;
    ltb_int_property(h, "bandwidth", &bw);
    int_properties["bandwidth"] = (int)bw;
    std::vector<char> buf(1 << 16);
    ltb_dump(h, buf.data(), buf.size());
    string_properties["code"] = buf.data();
  }
  ~B200Compiled() override { ltb_release(h); }
  void run(const std::vector<void*>& memory, bool sync) const override {
    int64_t tuned = 1;
    ltb_int_property(h, "tuned", &tuned);
    if (!tuned && autotune()) {
      // tuning needs device-visible buffers (managed memory from the "cuda"
      // hardware qualifies); it leaves the outputs computed
      if (ltb_tune(h, memory.data(), (int)memory.size(), nullptr, 5, nullptr, 0) == LTB_OK) {
        if (const char* f = schedule_file()) ltb_tune_save(f);
        if (sync) ltb_synchronize(nullptr);
        return;
      }
    }
    ASSERT(ltb_run(h, memory.data(), (int)memory.size(), sync ? 1 : 0, nullptr) == LTB_OK)
        << ltb_last_error();
  }
  std::string dump() const override { return string_properties.at("code"); }
};

struct B200Backend : public loop_tool::Backend {
  int hw_id;
  explicit B200Backend(int id) : Backend("cuda"), hw_id(id) {}
  std::unique_ptr<loop_tool::Compiled> compile_impl(
      const loop_tool::LoopTree& lt) const override {
    return std::make_unique<B200Compiled>(lt);
  }
  int hardware_requirement() const override { return 1 << hw_id; }
};

struct Registration {
  Registration() {
    if (ltb_device_count() == 0) return;
    if (const char* f = schedule_file()) ltb_tune_load(f);  // absent file: start empty
    auto hw = std::make_shared<B200Hardware>();
    loop_tool::registerHardware(hw);
    loop_tool::registerBackend(std::make_shared<B200Backend>(hw->id()));
  }
};
Registration registration;

}  // namespace
