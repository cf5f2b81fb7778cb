// tests/libm_device_check.cu -- runs the DEVICE build of ww3-gpu_b200/csrc/libm_dev.cuh on a B200
// and compares every result with this host's glibc. Usage: libm_device_check <function> <stride>;
// unary functions take every stride-th float bit pattern (stride 1 = all 2^32), powf and atan2f
// take 2^32 / stride seeded argument pairs. Prints "checked N mismatches M first <bits>". NaN
// results compare equal whatever their payload (the device's canonical NaN against glibc's).
#include <cuda_runtime.h>
#include <omp.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../ww3-gpu_b200/csrc/libm_dev.cuh"

namespace {

enum Fn { EXPF, LOGF, SINF, COSF, TANHF, ATANF, LOG10F, SINHF, COSHF, POWF, ATAN2F };

__host__ __device__ inline uint64_t mix(uint64_t i) {
  uint64_t h = i * 0x9E3779B97F4A7C15ULL;
  h ^= h >> 29;
  h *= 0xBF58476D1CE4E5B9ULL;
  h ^= h >> 32;
  return h;
}

__global__ void run(int fn, uint64_t first, long long n, long long stride, float* out) {
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < n;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const uint64_t idx = first + t;
    float r = 0.0f;
    if (fn < POWF) {
      const float x = __uint_as_float(static_cast<uint32_t>(idx * static_cast<uint64_t>(stride)));
      float s, c;
      switch (fn) {
        case EXPF: r = wwb::dm::expf(x); break;
        case LOGF: r = wwb::dm::logf(x); break;
        case SINF: wwb::dm::sincosf(x, &s, &c); r = s; break;
        case COSF: wwb::dm::sincosf(x, &s, &c); r = c; break;
        case TANHF: r = wwb::dm::tanhf(x); break;
        case ATANF: r = wwb::dm::atanf(x); break;
        case LOG10F: r = wwb::dm::log10f(x); break;
        case SINHF: r = wwb::dm::sinhf(x); break;
        default: r = wwb::dm::coshf(x); break;
      }
    } else {
      const uint64_t h = mix(idx);
      const float x = __uint_as_float(static_cast<uint32_t>(h));
      const float y = __uint_as_float(static_cast<uint32_t>(h >> 32));
      r = fn == POWF ? wwb::dm::powf(x, y) : wwb::dm::atan2f(y, x);
    }
    out[t] = r;
  }
}

float host_fn(int fn, uint64_t idx, long long stride) {
  if (fn < POWF) {
    uint32_t u = static_cast<uint32_t>(idx * static_cast<uint64_t>(stride));
    float x;
    std::memcpy(&x, &u, 4);
    float s, c;
    switch (fn) {
      case EXPF: return ::expf(x);
      case LOGF: return ::logf(x);
      case SINF: ::sincosf(x, &s, &c); return s;
      case COSF: ::sincosf(x, &s, &c); return c;
      case TANHF: return ::tanhf(x);
      case ATANF: return ::atanf(x);
      case LOG10F: return ::log10f(x);
      case SINHF: return ::sinhf(x);
      default: return ::coshf(x);
    }
  }
  const uint64_t h = mix(idx);
  const uint32_t ux = static_cast<uint32_t>(h), uy = static_cast<uint32_t>(h >> 32);
  float x, y;
  std::memcpy(&x, &ux, 4);
  std::memcpy(&y, &uy, 4);
  return fn == POWF ? ::powf(x, y) : ::atan2f(y, x);
}

}  // namespace

int main(int argc, char** argv) {
  const char* names[] = {"expf", "logf", "sinf", "cosf", "tanhf", "atanf", "log10f", "sinhf",
                         "coshf", "powf", "atan2f"};
  const char* want = argc > 1 ? argv[1] : "expf";
  const long long stride = argc > 2 ? std::atoll(argv[2]) : 1;
  int fn = -1;
  for (int i = 0; i < 11; ++i)
    if (std::strcmp(want, names[i]) == 0) fn = i;
  if (fn < 0 || stride < 1) {
    std::fprintf(stderr, "usage: libm_device_check <function> <stride>\n");
    return 2;
  }
  const long long total = (1LL << 32) / stride;
  const long long chunk = 1LL << 26;
  float* d = nullptr;
  if (cudaMalloc(&d, chunk * sizeof(float)) != cudaSuccess) return 3;
  std::vector<float> h(static_cast<size_t>(chunk));
  long long bad = 0;
  long long first_bad = -1;
  for (long long first = 0; first < total; first += chunk) {
    const long long n = (total - first < chunk) ? total - first : chunk;
    run<<<148 * 8, 256>>>(fn, static_cast<uint64_t>(first), n, stride, d);
    if (cudaMemcpy(h.data(), d, n * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) {
      std::fprintf(stderr, "CUDA error: %s\n", cudaGetErrorString(cudaGetLastError()));
      return 3;
    }
    long long b = 0, fb = -1;
#pragma omp parallel for reduction(+ : b) schedule(static)
    for (long long t = 0; t < n; ++t) {
      const float g = host_fn(fn, static_cast<uint64_t>(first + t), stride);
      const float r = h[static_cast<size_t>(t)];
      uint32_t ug, ur;
      std::memcpy(&ug, &g, 4);
      std::memcpy(&ur, &r, 4);
      if (ug != ur && !(std::isnan(g) && std::isnan(r))) {
        ++b;
#pragma omp critical
        if (fb < 0 || first + t < fb) fb = first + t;
      }
    }
    bad += b;
    if (fb >= 0 && first_bad < 0) first_bad = fb;
  }
  cudaFree(d);
  std::printf("%s checked %lld mismatches %lld first %lld\n", names[fn], total, bad, first_bad);
  return 0;
}
