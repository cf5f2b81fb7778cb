// ww3-gpu_b200/csrc/abi_core.cpp
// The runtime half of the C ABI: ww_kokkos_init / ww_kokkos_finalize, the run-time flags
// (ww_kokkos_flag and friends) and the WW_KOKKOS_TIMERS regions.
//
// Reference behaviour kept: ww_kokkos_init picks the device from WW_KOKKOS_DEVICE_ID and
// ignores the communicator (ww3-gpu kokkos/src/fortran_iface/ww_kokkos_c.hpp:52-73,
// snl1_shim.cpp:128-144, 196-237); the flag rules are those of part_flags.cpp (its behaviour, not its code); the
// timer totals print at exit in the format of timers.cpp:37-43.
#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <set>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "wwb_common.hpp"

namespace wwb {

Runtime& runtime() {
  static Runtime* r = new Runtime();  // never destroyed: finalize may run from atexit
  return *r;
}

void release_snl1_contexts();  // abi_snl1.cpp
void release_va_contexts();    // abi_va.cu
void release_prop3_staging();  // abi_prop3.cpp
void release_srce_contexts();  // abi_srce.cpp
void release_st4_contexts();   // abi_st4.cpp
void release_steps();          // abi_step.cpp
void release_outg_staging();   // abi_outg.cpp
void release_wave_staging();   // abi_wave.cpp
void release_sur_contexts();   // abi_sur.cpp

namespace {

Status g_core_status;
bool g_atexit_registered = false;

int device_id_from_env() {
  const char* v = std::getenv("WW_KOKKOS_DEVICE_ID");
  if (v == nullptr || *v == '\0') return 0;
  char* end = nullptr;
  const long id = std::strtol(v, &end, 10);
  if (end == v || *end != '\0' || id < 0 || id > 65535) {
    std::fprintf(stderr, "ww_b200: WW_KOKKOS_DEVICE_ID='%s' is not a device id; using 0\n", v);
    return 0;
  }
  return static_cast<int>(id);
}

// ---- run-time switches ---------------------------------------------------------------------
// The environment the WW3 fork's switch reads, resolved once per process: WW_KOKKOS_PRESET
// (a named set of parts, the reference's presets.txt), WW_KOKKOS_ALL and WW_KOKKOS_STRICT.
// A part's own variable WW_KOKKOS_<PART> is read at each ww_kokkos_flag call and wins over both.
bool is_one(const char* v) { return v != nullptr && v[0] == '1' && v[1] == '\0'; }

struct Switches {
  int preset = 0;                      // ww_kokkos_preset_status: 0 none, 1 known, -1 unknown
  std::set<std::string> preset_parts;  // parts the preset turns on, without the prefix
  bool all = false;
  bool strict = false;

  static const Switches& get() {
    static const Switches s = [] {
      // The presets of the reference (kokkos/src/fortran_iface/presets.txt), by name.
      static const std::map<std::string, std::set<std::string>> known = {
          {"resident", {"SRCE", "XYP3", "KTP3", "OUTG", "IOPE", "UPDV", "CPRT"}}};
      Switches x;
      const char* name = std::getenv("WW_KOKKOS_PRESET");
      if (name != nullptr && name[0] != '\0') {
        const auto it = known.find(name);
        x.preset = it == known.end() ? -1 : 1;
        if (it != known.end()) x.preset_parts = it->second;
      }
      x.all = is_one(std::getenv("WW_KOKKOS_ALL"));
      x.strict = is_one(std::getenv("WW_KOKKOS_STRICT"));
      return x;
    }();
    return s;
  }
};

/// Parts that only their own variable or a preset turns on: WW_KOKKOS_ALL leaves them off (the
/// reference's opt-in parts, kokkos/src/fortran_iface/part_flags.cpp:83-87).
bool opt_in_only(const std::string& part) {
  static const std::set<std::string> parts = {"XYP1", "KTP1", "XYP2", "KTP2", "XYPUG", "XYP3",
                                              "KTP3", "OUTG", "IOPE", "UPDV", "CPRT",
                                              "ST4_TABLES"};
  return parts.count(part) != 0;
}

/// Counters of calls a caller left on the Fortran, one per part, printed once at exit.
struct FallbackTally {
  static constexpr size_t kParts = 64;    // at most this many parts
  static constexpr size_t kNameMax = 24;  // characters of a part name
  std::vector<std::pair<std::string, long long>> parts;
  static FallbackTally& get() {
    static auto* t = new FallbackTally();
    return *t;
  }
  static void print() {
    std::string line = "ww_b200: Fortran fallbacks by part (WW_KOKKOS_STRICT=1 stops instead):";
    for (const auto& [name, n] : get().parts) line += " " + name + "=" + std::to_string(n);
    std::fprintf(stderr, "%s\n", line.c_str());
  }
};

// ---- timers -----------------------------------------------------------------------------
struct Total {
  long long calls = 0;
  double seconds = 0.0;
};
std::mutex& timer_mu() {
  static auto* m = new std::mutex();
  return *m;
}
std::map<std::string, Total>& timer_totals() {
  static auto* m = new std::map<std::string, Total>();
  return *m;
}
void print_timers() {
  std::lock_guard<std::mutex> lock(timer_mu());
  for (const auto& [name, t] : timer_totals())
    std::fprintf(stderr, "ww_b200: time %s: %lld calls, %.6f s\n", name.c_str(), t.calls,
                 t.seconds);
}
double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

}  // namespace

namespace timers {
bool enabled() {
  static const bool on = [] {
    const char* v = std::getenv("WW_KOKKOS_TIMERS");
    return v != nullptr && std::strcmp(v, "1") == 0;
  }();
  return on;
}
void add(const char* name, double seconds) {
  std::lock_guard<std::mutex> lock(timer_mu());
  static bool registered = false;
  if (!registered) {
    std::atexit(print_timers);
    registered = true;
  }
  Total& t = timer_totals()[name];
  t.calls += 1;
  t.seconds += seconds;
}
// A region synchronises the device at its start and stop when timers are on, so its time is
// the work and not the launch (timers.hpp:3-6); off, it is one branch.
Region::Region(const char* name) : name_(name), on_(enabled()) {
  if (!on_) return;
  cudaDeviceSynchronize();
  t0_ = now_s();
}
void Region::stop() {
  if (!on_) return;
  on_ = false;
  cudaDeviceSynchronize();
  add(name_, now_s() - t0_);
}
}  // namespace timers

}  // namespace wwb

using wwb::runtime;

extern "C" {

int ww_kokkos_init(int comm_f) {
  (void)comm_f;  // the device comes from WW_KOKKOS_DEVICE_ID, as in the reference
  try {
    auto& rt = runtime();
    if (rt.ready) return WW_KOKKOS_OK;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
      cudaGetLastError();
      return wwb::g_core_status.fail(WW_KOKKOS_ERR_RUNTIME, "ww_kokkos_init: no CUDA device");
    }
    const int dev = wwb::device_id_from_env();
    if (dev >= ndev)
      return wwb::g_core_status.fail(WW_KOKKOS_ERR_RUNTIME,
                                     "ww_kokkos_init: WW_KOKKOS_DEVICE_ID beyond the devices");
    WWB_CHECK(cudaSetDevice(dev));
    WWB_CHECK(cudaFree(nullptr));  // create the context now, not inside the first call
    int sms = 0;
    WWB_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    WWB_CHECK(cudaStreamCreateWithFlags(&rt.stream, cudaStreamNonBlocking));
    WWB_CHECK(cudaStreamCreateWithFlags(&rt.copy_in, cudaStreamNonBlocking));
    WWB_CHECK(cudaStreamCreateWithFlags(&rt.copy_out, cudaStreamNonBlocking));
    rt.device = dev;
    rt.sm_count = sms;
    rt.ready = true;
    if (!wwb::g_atexit_registered) {
      std::atexit(ww_kokkos_finalize);
      wwb::g_atexit_registered = true;
    }
    wwb::g_core_status.ok();
    return WW_KOKKOS_OK;
  } catch (const std::exception& e) {
    return wwb::g_core_status.fail(WW_KOKKOS_ERR_RUNTIME, e.what());
  }
}

void ww_kokkos_finalize(void) {
  auto& rt = runtime();
  wwb::release_steps();
  wwb::release_sur_contexts();
  wwb::release_srce_contexts();
  wwb::release_st4_contexts();
  wwb::release_snl1_contexts();
  if (!rt.ready) return;
  wwb::release_va_contexts();
  wwb::release_prop3_staging();
  wwb::release_outg_staging();
  wwb::release_wave_staging();
  cudaDeviceSynchronize();
  if (rt.stream) cudaStreamDestroy(rt.stream);
  if (rt.copy_in) cudaStreamDestroy(rt.copy_in);
  if (rt.copy_out) cudaStreamDestroy(rt.copy_out);
  rt.stream = rt.copy_in = rt.copy_out = nullptr;
  rt.ready = false;
}

int ww_kokkos_flag(const char* name) {
  if (name == nullptr) return 0;
  if (const char* own = std::getenv(name)) return wwb::is_one(own) ? 1 : 0;
  const wwb::Switches& sw = wwb::Switches::get();
  const std::string full(name), prefix("WW_KOKKOS_");
  if (full.compare(0, prefix.size(), prefix) == 0) {
    const std::string part = full.substr(prefix.size());
    if (sw.preset_parts.count(part) != 0) return 1;
    if (wwb::opt_in_only(part)) return 0;
  }
  return sw.all ? 2 : 0;
}

int ww_kokkos_preset_status(void) { return wwb::Switches::get().preset; }

int ww_kokkos_strict(void) { return wwb::Switches::get().strict ? 1 : 0; }

int ww_kokkos_fallback_slot(const char* part) {
  using wwb::FallbackTally;
  if (part == nullptr || std::strlen(part) > FallbackTally::kNameMax) return -1;
  auto& parts = FallbackTally::get().parts;
  for (size_t i = 0; i < parts.size(); ++i)
    if (parts[i].first == part) return static_cast<int>(i);
  if (parts.size() == FallbackTally::kParts) return -1;
  if (parts.empty()) std::atexit(FallbackTally::print);
  parts.emplace_back(part, 0);
  return static_cast<int>(parts.size() - 1);
}

void ww_kokkos_fallback_add(int slot) {
  auto& parts = wwb::FallbackTally::get().parts;
  if (slot >= 0 && static_cast<size_t>(slot) < parts.size()) ++parts[slot].second;
}

}  // extern "C"
