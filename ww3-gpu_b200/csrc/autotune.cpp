// ww3-gpu_b200/csrc/autotune.cpp -- see autotune.hpp.
#include "autotune.hpp"

#include <algorithm>
#include <cstdio>
#include <map>
#include <utility>

#include "wwb_common.hpp"

namespace wwb {
namespace tune {
namespace {

struct Record {
  int choice = 0;
  std::vector<std::pair<int, float>> ms;  // candidate, median ms
};

std::map<std::string, Record>& records() {
  static auto* m = new std::map<std::string, Record>();
  return *m;
}

}  // namespace

int pick(const std::string& key, const std::vector<int>& cands,
         const std::function<void(int, cudaStream_t)>& run,
         const std::function<void(int, cudaStream_t)>& prepare, cudaStream_t st, int reps) {
  if (cands.empty()) throw CudaError(cudaErrorInvalidValue, "autotune: no candidate");
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  WWB_CHECK(cudaEventCreate(&e0));
  WWB_CHECK(cudaEventCreate(&e1));
  Record rec;
  float best = 0.0f;
  try {
    for (int c : cands) {
      if (prepare) prepare(c, st);
      run(c, st);  // warm-up: first-launch set-up, caches
      std::vector<float> t;
      for (int r = 0; r < reps; ++r) {
        if (prepare) prepare(c, st);
        WWB_CHECK(cudaEventRecord(e0, st));
        run(c, st);
        WWB_CHECK(cudaEventRecord(e1, st));
        WWB_CHECK(cudaEventSynchronize(e1));
        float ms = 0.0f;
        WWB_CHECK(cudaEventElapsedTime(&ms, e0, e1));
        t.push_back(ms);
      }
      std::sort(t.begin(), t.end());
      const float med = t[t.size() / 2];
      rec.ms.emplace_back(c, med);
      if (rec.ms.size() == 1 || med < best) {
        best = med;
        rec.choice = c;
      }
    }
  } catch (...) {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  records()[key] = rec;
  return rec.choice;
}

int cached(const std::string& key, int fallback) {
  auto it = records().find(key);
  return it == records().end() ? fallback : it->second.choice;
}

std::string device_key() {
  int dev = 0;
  WWB_CHECK(cudaGetDevice(&dev));
  cudaDeviceProp p{};
  WWB_CHECK(cudaGetDeviceProperties(&p, dev));
  char b[64];
  std::snprintf(b, sizeof b, "sm%d%d x%d dev%d", p.major, p.minor, p.multiProcessorCount, dev);
  return b;
}

std::string report() {
  std::string s = "{";
  bool first = true;
  for (const auto& kv : records()) {
    if (!first) s += ", ";
    first = false;
    char b[64];
    std::snprintf(b, sizeof b, "%d", kv.second.choice);
    s += "\"" + kv.first + "\": {\"choice\": " + b + ", \"ms\": {";
    bool f2 = true;
    for (const auto& cm : kv.second.ms) {
      char c[64];
      std::snprintf(c, sizeof c, "%s\"%d\": %.4f", f2 ? "" : ", ", cm.first, cm.second);
      s += c;
      f2 = false;
    }
    s += "}}";
  }
  return s + "}";
}

}  // namespace tune
}  // namespace wwb

extern "C" int ww_autotune_report(char* buf, int len) {
  try {
    const std::string r = wwb::tune::report();
    if (buf != nullptr && len > 0) {
      const size_t n = std::min(r.size(), static_cast<size_t>(len - 1));
      std::copy(r.begin(), r.begin() + n, buf);
      buf[n] = '\0';
    }
    return static_cast<int>(r.size());
  } catch (...) {
    return -1;
  }
}
