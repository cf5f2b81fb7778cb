// ww3-gpu_b200/csrc/abi_core.cpp
// The runtime half of the C ABI: ww_kokkos_init / ww_kokkos_finalize, the run-time flags
// (ww_kokkos_flag and friends) and the WW_KOKKOS_TIMERS regions.
//
// Reference behaviour kept: ww_kokkos_init picks the device from WW_KOKKOS_DEVICE_ID and
// ignores the communicator (ww3-gpu kokkos/src/fortran_iface/ww_kokkos_c.hpp:52-73,
// snl1_shim.cpp:128-144, 196-237); the flag rules are those of part_flags.cpp:1-135; the
// timer totals print at exit in the format of timers.cpp:37-43.
#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>

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

// ---- run-time flags -------------------------------------------------------------------
struct Preset {
  const char* name;
  const char* parts;
};
// The reference's one preset (kokkos/src/fortran_iface/presets.txt).
constexpr Preset kPresets[] = {{"resident", "SRCE,XYP3,KTP3,OUTG,IOPE,UPDV,CPRT"}};
constexpr Preset kUnknown{"", ""};
// Parts that WW_KOKKOS_ALL does not turn on (part_flags.cpp:60-64).
constexpr const char* kOptInOnly[] = {"WW_KOKKOS_XYP1", "WW_KOKKOS_KTP1", "WW_KOKKOS_XYP2",
                                      "WW_KOKKOS_KTP2", "WW_KOKKOS_XYPUG", "WW_KOKKOS_XYP3",
                                      "WW_KOKKOS_KTP3", "WW_KOKKOS_OUTG", "WW_KOKKOS_IOPE",
                                      "WW_KOKKOS_UPDV", "WW_KOKKOS_CPRT",
                                      "WW_KOKKOS_ST4_TABLES"};

const Preset* preset() {
  static const Preset* const p = []() -> const Preset* {
    const char* v = std::getenv("WW_KOKKOS_PRESET");
    if (v == nullptr || *v == '\0') return nullptr;
    for (const Preset& q : kPresets)
      if (std::strcmp(v, q.name) == 0) return &q;
    return &kUnknown;
  }();
  return p;
}

bool in_list(const char* part, const char* list) {
  const size_t n = std::strlen(part);
  const char* s = list;
  while (*s != '\0') {
    const char* e = std::strchr(s, ',');
    const size_t m = e ? static_cast<size_t>(e - s) : std::strlen(s);
    if (m == n && std::strncmp(s, part, n) == 0) return true;
    if (e == nullptr) break;
    s = e + 1;
  }
  return false;
}

constexpr int kMaxSlots = 64;
char g_slot_name[kMaxSlots][25] = {};
long long g_slot_count[kMaxSlots] = {};
int g_nslots = 0;

void print_fallbacks() {
  std::fprintf(stderr, "ww_b200: calls left on the Fortran (WW_KOKKOS_STRICT=1 stops instead):");
  for (int i = 0; i < g_nslots; ++i)
    std::fprintf(stderr, " %s=%lld", g_slot_name[i], g_slot_count[i]);
  std::fprintf(stderr, "\n");
}

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
  if (const char* v = std::getenv(name)) return std::strcmp(v, "1") == 0 ? 1 : 0;
  constexpr const char kPrefix[] = "WW_KOKKOS_";
  const wwb::Preset* p = wwb::preset();
  if (p != nullptr && std::strncmp(name, kPrefix, sizeof kPrefix - 1) == 0 &&
      wwb::in_list(name + sizeof kPrefix - 1, p->parts))
    return 1;
  for (const char* q : wwb::kOptInOnly)
    if (std::strcmp(name, q) == 0) return 0;
  const char* all = std::getenv("WW_KOKKOS_ALL");
  return (all != nullptr && std::strcmp(all, "1") == 0) ? 2 : 0;
}

int ww_kokkos_preset_status(void) {
  const wwb::Preset* p = wwb::preset();
  return p == nullptr ? 0 : (p == &wwb::kUnknown ? -1 : 1);
}

int ww_kokkos_strict(void) {
  static const int strict = [] {
    const char* v = std::getenv("WW_KOKKOS_STRICT");
    return (v != nullptr && std::strcmp(v, "1") == 0) ? 1 : 0;
  }();
  return strict;
}

int ww_kokkos_fallback_slot(const char* part) {
  if (part == nullptr || std::strlen(part) >= sizeof wwb::g_slot_name[0]) return -1;
  for (int i = 0; i < wwb::g_nslots; ++i)
    if (std::strcmp(wwb::g_slot_name[i], part) == 0) return i;
  if (wwb::g_nslots == wwb::kMaxSlots) return -1;
  if (wwb::g_nslots == 0) std::atexit(wwb::print_fallbacks);
  std::strcpy(wwb::g_slot_name[wwb::g_nslots], part);
  return wwb::g_nslots++;
}

void ww_kokkos_fallback_add(int slot) {
  if (slot >= 0 && slot < wwb::g_nslots) ++wwb::g_slot_count[slot];
}

}  // extern "C"
