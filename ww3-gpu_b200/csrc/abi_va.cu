// ww3-gpu_b200/csrc/abi_va.cu
// The resident spectrum behind the ww_va_* entries: one ResidentVa object per grid, a small
// state machine over which copy of VA(NSPEC, 0:NSEALM) holds the newer bits.
//
// The contract is the reference ABI's (ww3-gpu kokkos/src/fortran_iface/resident_c.hpp:10-101):
// bind to the caller's VA on the grid's first call and refuse another address or shape; the
// state (HOST, DEVICE, BOTH, the values ww_va_state returns) changes only as the table below
// says; partial reads and writes of listed columns cross packed and leave the state alone; the
// WW_KOKKOS_VA_RESIDENT / _CHECK / _POISON / _COUNT diagnostics. The implementation is this
// library's own:
//
//   event (entry)                      HOST          DEVICE                BOTH
//   host read (ww_va_host_read)        -             download -> BOTH      -
//   host write (ww_va_host_write)      -             download -> HOST      -> HOST
//   kernel sync (ww_va_device, write)  upload->BOTH  -                     -       (then DEVICE)
//   partial read (_read_cols)          -             gather listed cols    -
//   partial write (_wrote_cols)        -             scatter listed cols   scatter listed cols
//   host zeroed cols (_device_zero)    -             zero listed on device zero listed on device
//
// Every transition is a member of ResidentVa; copies move bits and compute nothing. Packed
// columns go through one staging area per grid (device index and value buffers and a
// page-locked host buffer, grown to the largest list seen) instead of per-list buffers.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <new>
#include <vector>

#include "va.hpp"
#include "wwb_common.hpp"

namespace wwb {
namespace {

enum VaState : int { kHost = 0, kDevice = 1, kBoth = 2 };  // ww_va_state's values

/// The diagnostics switches, read from the environment once per process.
struct Diagnostics {
  bool resident = false;  ///< WW_KOKKOS_VA_RESIDENT=1: every host call round-trips d_va
  bool audit = false;     ///< WW_KOKKOS_VA_CHECK=1: compare bits against the last sync
  bool poison = false;    ///< WW_KOKKOS_VA_POISON=1: NaN-fill the stale host VA
  bool tally = false;     ///< WW_KOKKOS_VA_COUNT=1: print the traffic at exit
  static const Diagnostics& get() {
    static const Diagnostics d = [] {
      auto on = [](const char* name) {
        const char* v = std::getenv(name);
        return v != nullptr && v[0] == '1' && v[1] == '\0';
      };
      Diagnostics x;
      x.resident = on("WW_KOKKOS_VA_RESIDENT");
      x.audit = on("WW_KOKKOS_VA_CHECK");
      x.poison = on("WW_KOKKOS_VA_POISON");
      x.tally = on("WW_KOKKOS_VA_COUNT");
      return x;
    }();
    return d;
  }
};

/// What crossed, for ww_va_report.
struct Traffic {
  long long uploads = 0, downloads = 0;                  // whole-array copies
  double upload_mb = 0, download_mb = 0;
  long long host_syncs = 0, kernel_syncs = 0;            // entry calls
  long long col_reads = 0, col_read_copies = 0, col_read_columns = 0;
  long long col_writes = 0, col_write_copies = 0, col_write_columns = 0;
  double col_mb = 0;
  long long updates = 0, zero_launches = 0, zero_columns = 0;
  long long audits = 0, poisonings = 0;
};
Traffic g_traffic;

void report_line(const char* text) { std::fprintf(stderr, "ww_b200 [va] %s\n", text); }

/// The quiet NaN written over a stale host VA under WW_KOKKOS_VA_POISON=1.
constexpr uint32_t kPoisonBits = 0x7FC0FA11u;

__global__ void pack_kernel(const float* __restrict__ va, const int* __restrict__ cols, int ncol,
                            int nspec, float* __restrict__ packed) {
  const size_t total = static_cast<size_t>(ncol) * nspec;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<size_t>(gridDim.x) * blockDim.x)
    packed[i] = va[static_cast<size_t>(cols[i / nspec]) * nspec + i % nspec];
}

__global__ void unpack_kernel(float* __restrict__ va, const int* __restrict__ cols, int ncol,
                              int nspec, const float* __restrict__ packed) {
  const size_t total = static_cast<size_t>(ncol) * nspec;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<size_t>(gridDim.x) * blockDim.x)
    va[static_cast<size_t>(cols[i / nspec]) * nspec + i % nspec] = packed[i];
}

__global__ void clear_kernel(float* __restrict__ va, const int* __restrict__ cols, int ncol,
                             int nspec) {
  const size_t total = static_cast<size_t>(ncol) * nspec;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<size_t>(gridDim.x) * blockDim.x)
    va[static_cast<size_t>(cols[i / nspec]) * nspec + i % nspec] = 0.0f;
}

unsigned blocks_for(size_t n) {
  const size_t want = (n + 255) / 256;
  const size_t most = static_cast<size_t>(runtime().sm_count > 0 ? runtime().sm_count : 148) * 8;
  return static_cast<unsigned>(std::max<size_t>(1, std::min(want, most)));
}

/// A column list as the entries receive it, validated: sorted, duplicates removed.
struct ColumnList {
  std::vector<int> jsea;
  bool valid = true;
  ColumnList(int n, const int* cols, int nsealm, bool dedupe) {
    if (n < 0 || (n > 0 && cols == nullptr)) {
      valid = false;
      return;
    }
    jsea.assign(cols, cols + n);
    for (const int j : jsea)
      if (j < 0 || j > nsealm) valid = false;
    if (dedupe) {
      std::sort(jsea.begin(), jsea.end());
      jsea.erase(std::unique(jsea.begin(), jsea.end()), jsea.end());
    }
  }
  int size() const { return static_cast<int>(jsea.size()); }
};

class ResidentVa {
 public:
  ResidentVa() = default;
  ResidentVa(const ResidentVa&) = delete;
  ResidentVa& operator=(const ResidentVa&) = delete;
  ~ResidentVa() { release(); }

  /// Binds on the first call; later calls must pass the same array. Returns a status.
  int attach(int igrid, float* va, int nspec, int nsealm) {
    if (va == nullptr || nspec <= 0 || nsealm < 0) {
      report_line("refused: a null VA or a negative extent");
      return WW_KOKKOS_ERR_BAD_SHAPE;
    }
    if (host_ == nullptr) {
      igrid_ = igrid;
      host_ = va;
      nspec_ = nspec;
      ncols_ = static_cast<size_t>(nsealm) + 1;
      return WW_KOKKOS_OK;
    }
    if (host_ == va && nspec_ == nspec && ncols_ == static_cast<size_t>(nsealm) + 1)
      return WW_KOKKOS_OK;
    std::fprintf(stderr,
                 "ww_b200 [va] grid %d is bound to VA at %p (%d x 0:%zu); a call passed %p "
                 "(%d x 0:%d): one VA per grid\n",
                 igrid, static_cast<void*>(host_), nspec_, ncols_ - 1, static_cast<void*>(va),
                 nspec, nsealm);
    return WW_KOKKOS_ERR_BAD_SHAPE;
  }

  VaState state() const { return state_; }
  float* device() const { return dev_; }
  bool bound() const { return host_ != nullptr; }

  /// Before the host reads (writes == false) or writes the whole VA.
  int host_access(bool writes) {
    if (int rc = audit(writes ? "host write" : "host read"); rc != WW_KOKKOS_OK) return rc;
    ++g_traffic.host_syncs;
    if (Diagnostics::get().resident) {
      if (!runtime().ready) return WW_KOKKOS_ERR_NOT_INITIALISED;
      if (state_ == kHost) upload();
      download();
    } else if (state_ == kDevice) {
      download();
    }
    if (writes) {
      state_ = kHost;
      shadow_valid_ = false;
    }
    return WW_KOKKOS_OK;
  }

  /// Before a kernel reads d_va; with `writes` the device copy is the newer one afterwards.
  int kernel_access(bool writes) {
    if (int rc = audit("kernel sync"); rc != WW_KOKKOS_OK) return rc;
    ++g_traffic.kernel_syncs;
    if (state_ == kHost) upload();
    if (writes) state_ = kDevice;
    return WW_KOKKOS_OK;
  }

  /// A kernel wrote d_va (the caller launched it after kernel_access).
  void kernel_wrote() {
    if (dev_ == nullptr) return;
    state_ = kDevice;
    if (Diagnostics::get().poison) {
      float nan;
      std::memcpy(&nan, &kPoisonBits, sizeof nan);
      std::fill_n(host_, count(), nan);
      shadow_valid_ = false;
      ++g_traffic.poisonings;
    }
  }

  /// The host is about to read the listed columns only.
  int read_columns(const ColumnList& c) {
    if (int rc = audit("partial host read"); rc != WW_KOKKOS_OK) return rc;
    ++g_traffic.col_reads;
    if (Diagnostics::get().resident) {
      if (!runtime().ready) return WW_KOKKOS_ERR_NOT_INITIALISED;
      if (state_ == kHost) upload();
    } else if (state_ != kDevice) {
      return WW_KOKKOS_OK;  // the host copy is current
    }
    if (c.size() == 0) return WW_KOKKOS_OK;
    stage(c);
    const size_t n = static_cast<size_t>(c.size()) * nspec_;
    {
      timers::Region t("va.cols_to_host");
      WWB_CHECK(cudaDeviceSynchronize());  // kernels on other streams may have written d_va
      pack_kernel<<<blocks_for(n), 256>>>(dev_, d_idx_, c.size(), nspec_, d_pack_);
      WWB_CHECK(cudaGetLastError());
      WWB_CHECK(cudaMemcpy(h_pack_, d_pack_, n * sizeof(float), cudaMemcpyDeviceToHost));
    }
    for (int k = 0; k < c.size(); ++k) {
      std::memcpy(column(host_, c.jsea[k]), h_pack_ + k * static_cast<size_t>(nspec_), col_bytes());
      if (shadow_valid_) std::memcpy(column(shadow_.data(), c.jsea[k]), h_pack_ + k * static_cast<size_t>(nspec_), col_bytes());
    }
    ++g_traffic.col_read_copies;
    g_traffic.col_read_columns += c.size();
    g_traffic.col_mb += n * 4e-6;
    return WW_KOKKOS_OK;
  }

  /// The host wrote the listed columns (and no other).
  int wrote_columns(const ColumnList& c) {
    if (shadow_valid_)
      for (const int j : c.jsea) std::memcpy(column(shadow_.data(), j), column(host_, j), col_bytes());
    if (int rc = audit("partial host write"); rc != WW_KOKKOS_OK) return rc;
    ++g_traffic.col_writes;
    if (state_ == kHost || c.size() == 0) {
      if (Diagnostics::get().resident && state_ == kHost) {
        if (!runtime().ready) return WW_KOKKOS_ERR_NOT_INITIALISED;
        upload();
      }
      return WW_KOKKOS_OK;
    }
    if (!runtime().ready) return WW_KOKKOS_ERR_NOT_INITIALISED;
    stage(c);
    for (int k = 0; k < c.size(); ++k)
      std::memcpy(h_pack_ + k * static_cast<size_t>(nspec_), column(host_, c.jsea[k]), col_bytes());
    const size_t n = static_cast<size_t>(c.size()) * nspec_;
    {
      timers::Region t("va.cols_to_device");
      WWB_CHECK(cudaDeviceSynchronize());
      WWB_CHECK(cudaMemcpy(d_pack_, h_pack_, n * sizeof(float), cudaMemcpyHostToDevice));
      unpack_kernel<<<blocks_for(n), 256>>>(dev_, d_idx_, c.size(), nspec_, d_pack_);
      WWB_CHECK(cudaGetLastError());
      WWB_CHECK(cudaDeviceSynchronize());
    }
    ++g_traffic.col_write_copies;
    g_traffic.col_write_columns += c.size();
    g_traffic.col_mb += n * 4e-6;
    if (Diagnostics::get().resident) download();
    return WW_KOKKOS_OK;
  }

  /// The host zeroed the listed columns; repeat it on d_va unless the host copy is the newer.
  int zero_columns(const ColumnList& c) {
    if (state_ == kHost) return WW_KOKKOS_OK;
    if (!runtime().ready) return WW_KOKKOS_ERR_NOT_INITIALISED;
    if (c.size() > 0) {
      stage(c);
      const size_t n = static_cast<size_t>(c.size()) * nspec_;
      WWB_CHECK(cudaDeviceSynchronize());
      clear_kernel<<<blocks_for(n), 256>>>(dev_, d_idx_, c.size(), nspec_);
      WWB_CHECK(cudaGetLastError());
      WWB_CHECK(cudaDeviceSynchronize());
      ++g_traffic.zero_launches;
      g_traffic.zero_columns += c.size();
      if (shadow_valid_)
        for (const int j : c.jsea) std::fill_n(column(shadow_.data(), j), nspec_, 0.0f);
    }
    if (Diagnostics::get().resident) {
      // ww_va_host_update made both copies equal; a zeroed column the list missed shows here.
      std::vector<float> dev_bits(count());
      WWB_CHECK(cudaMemcpy(dev_bits.data(), dev_, bytes(), cudaMemcpyDeviceToHost));
      const long long bad = differing_columns(dev_bits.data(), host_);
      if (bad != 0) {
        std::fprintf(stderr,
                     "ww_b200 [va] grid %d: after zeroing, %lld columns of d_va differ from the "
                     "host VA (a column the host zeroed is missing from the list)\n",
                     igrid_, bad);
        return WW_KOKKOS_ERR_KERNEL;
      }
    }
    return WW_KOKKOS_OK;
  }

  /// ww_va_host_update: no copy unless WW_KOKKOS_VA_RESIDENT=1, then a host read.
  int host_update() {
    ++g_traffic.updates;
    if (!Diagnostics::get().resident) return audit("host update");
    return host_access(false);
  }

  void release() {
    if (state_ == kDevice && host_ != nullptr)
      std::fprintf(stderr, "ww_b200 [va] grid %d: the device copy was the newer one at finalize\n",
                   igrid_);
    if (dev_) cudaFree(dev_);
    if (d_idx_) cudaFree(d_idx_);
    if (d_pack_) cudaFree(d_pack_);
    if (h_pack_) cudaFreeHost(h_pack_);
    dev_ = d_pack_ = h_pack_ = nullptr;
    d_idx_ = nullptr;
    idx_cap_ = pack_cap_ = 0;
  }

 private:
  size_t count() const { return ncols_ * static_cast<size_t>(nspec_); }
  size_t bytes() const { return count() * sizeof(float); }
  size_t col_bytes() const { return static_cast<size_t>(nspec_) * sizeof(float); }
  float* column(float* base, int j) const { return base + static_cast<size_t>(j) * nspec_; }

  void upload() {
    if (dev_ == nullptr) WWB_CHECK(cudaMalloc(&dev_, bytes()));
    timers::Region t("va.to_device");
    WWB_CHECK(cudaMemcpy(dev_, host_, bytes(), cudaMemcpyHostToDevice));
    ++g_traffic.uploads;
    g_traffic.upload_mb += bytes() * 1e-6;
    state_ = kBoth;
    remember();
  }

  void download() {
    timers::Region t("va.to_host");
    WWB_CHECK(cudaDeviceSynchronize());  // the kernels that wrote d_va may be on any stream
    WWB_CHECK(cudaMemcpy(host_, dev_, bytes(), cudaMemcpyDeviceToHost));
    ++g_traffic.downloads;
    g_traffic.download_mb += bytes() * 1e-6;
    state_ = kBoth;
    remember();
  }

  /// Under WW_KOKKOS_VA_CHECK: the host bits at the latest sync.
  void remember() {
    if (!Diagnostics::get().audit) return;
    shadow_.assign(host_, host_ + count());
    shadow_valid_ = true;
  }

  long long differing_columns(const float* a, const float* b) const {
    long long n = 0;
    for (size_t j = 0; j < ncols_; ++j)
      if (std::memcmp(a + j * nspec_, b + j * nspec_, col_bytes()) != 0) ++n;
    return n;
  }

  /// Under WW_KOKKOS_VA_CHECK: unless the host copy is the newer one, the host VA must still hold
  /// the bits of the last sync; with both copies claimed equal, d_va must hold them too.
  int audit(const char* event) {
    if (!Diagnostics::get().audit || !shadow_valid_ || state_ == kHost) return WW_KOKKOS_OK;
    ++g_traffic.audits;
    if (const long long bad = differing_columns(host_, shadow_.data()); bad != 0) {
      std::fprintf(stderr,
                   "ww_b200 [va] WW_KOKKOS_VA_CHECK: grid %d at a %s: the host VA changed since "
                   "the last sync in %lld columns, with no host write declared\n",
                   igrid_, event, bad);
      return WW_KOKKOS_ERR_KERNEL;
    }
    if (state_ == kBoth && dev_ != nullptr) {
      std::vector<float> dev_bits(count());
      WWB_CHECK(cudaMemcpy(dev_bits.data(), dev_, bytes(), cudaMemcpyDeviceToHost));
      if (const long long bad = differing_columns(dev_bits.data(), shadow_.data()); bad != 0) {
        std::fprintf(stderr,
                     "ww_b200 [va] WW_KOKKOS_VA_CHECK: grid %d at a %s: d_va differs from the "
                     "host VA in %lld columns while both are marked equal\n",
                     igrid_, event, bad);
        return WW_KOKKOS_ERR_KERNEL;
      }
    }
    return WW_KOKKOS_OK;
  }

  /// The column list on the device and room for its packed values, grown on demand.
  void stage(const ColumnList& c) {
    const size_t ni = static_cast<size_t>(c.size());
    const size_t nv = ni * nspec_;
    if (ni > idx_cap_) {
      if (d_idx_) cudaFree(d_idx_);
      d_idx_ = nullptr;
      WWB_CHECK(cudaMalloc(&d_idx_, ni * sizeof(int)));
      idx_cap_ = ni;
    }
    if (nv > pack_cap_) {
      if (d_pack_) cudaFree(d_pack_);
      if (h_pack_) cudaFreeHost(h_pack_);
      d_pack_ = h_pack_ = nullptr;
      WWB_CHECK(cudaMalloc(&d_pack_, nv * sizeof(float)));
      WWB_CHECK(cudaMallocHost(&h_pack_, nv * sizeof(float)));
      pack_cap_ = nv;
    }
    WWB_CHECK(cudaMemcpy(d_idx_, c.jsea.data(), ni * sizeof(int), cudaMemcpyHostToDevice));
  }

  int igrid_ = 0;
  float* host_ = nullptr;
  int nspec_ = 0;
  size_t ncols_ = 0;
  float* dev_ = nullptr;
  VaState state_ = kHost;
  std::vector<float> shadow_;
  bool shadow_valid_ = false;
  int* d_idx_ = nullptr;
  float* d_pack_ = nullptr;
  float* h_pack_ = nullptr;
  size_t idx_cap_ = 0, pack_cap_ = 0;
};

std::map<int, ResidentVa>& registry() {
  static auto* m = new std::map<int, ResidentVa>();
  return *m;
}

/// The grid's object bound to (va, nspec, nsealm), or a status.
int bound_va(int igrid, float* va, int nspec, int nsealm, ResidentVa** out) {
  static bool report_at_exit = false;
  if (!report_at_exit && Diagnostics::get().tally) {
    std::atexit(ww_va_report);
    report_at_exit = true;
  }
  ResidentVa& r = registry()[igrid];
  const int rc = r.attach(igrid, va, nspec, nsealm);
  *out = rc == WW_KOKKOS_OK ? &r : nullptr;
  return rc;
}

/// Runs an entry's body; a CUDA failure or an allocation failure becomes a status.
template <class Body>
int as_status(Body&& body) {
  try {
    return body();
  } catch (const std::bad_alloc& e) {
    report_line(e.what());
    return WW_KOKKOS_ERR_RUNTIME;
  } catch (const std::exception& e) {
    report_line(e.what());
    return WW_KOKKOS_ERR_KERNEL;
  }
}

}  // namespace

int va_device(int igrid, float* va, int nspec, int nsealm, float** d_va) {
  return as_status([&]() {
    if (!runtime().ready) return static_cast<int>(WW_KOKKOS_ERR_NOT_INITIALISED);
    ResidentVa* r = nullptr;
    if (int rc = bound_va(igrid, va, nspec, nsealm, &r); rc != WW_KOKKOS_OK) return rc;
    if (int rc = r->kernel_access(false); rc != WW_KOKKOS_OK) return rc;
    *d_va = r->device();
    return static_cast<int>(WW_KOKKOS_OK);
  });
}

void va_device_written(int igrid) {
  auto it = registry().find(igrid);
  if (it != registry().end()) it->second.kernel_wrote();
}

int va_device_current(int igrid) {
  return as_status([&]() {
    auto it = registry().find(igrid);
    if (it == registry().end()) return static_cast<int>(WW_KOKKOS_OK);
    return it->second.kernel_access(true);
  });
}

void release_va_contexts() { registry().clear(); }

}  // namespace wwb

using namespace wwb;

extern "C" {

int ww_va_host_read(int igrid, float* va, int nspec, int nsealm) {
  return as_status([&]() {
    ResidentVa* r = nullptr;
    if (int rc = bound_va(igrid, va, nspec, nsealm, &r); rc != WW_KOKKOS_OK) return rc;
    return r->host_access(false);
  });
}

int ww_va_host_write(int igrid, float* va, int nspec, int nsealm) {
  return as_status([&]() {
    ResidentVa* r = nullptr;
    if (int rc = bound_va(igrid, va, nspec, nsealm, &r); rc != WW_KOKKOS_OK) return rc;
    return r->host_access(true);
  });
}

int ww_va_host_read_cols(int igrid, float* va, int nspec, int nsealm, int ncol,
                         const int* cols) {
  return as_status([&]() {
    ResidentVa* r = nullptr;
    if (int rc = bound_va(igrid, va, nspec, nsealm, &r); rc != WW_KOKKOS_OK) return rc;
    const ColumnList c(ncol, cols, nsealm, true);
    if (!c.valid) {
      report_line("ww_va_host_read_cols refused: a column outside 0..NSEALM or a null list");
      return static_cast<int>(WW_KOKKOS_ERR_BAD_SHAPE);
    }
    return r->read_columns(c);
  });
}

int ww_va_host_wrote_cols(int igrid, float* va, int nspec, int nsealm, int ncol,
                          const int* cols) {
  return as_status([&]() {
    ResidentVa* r = nullptr;
    if (int rc = bound_va(igrid, va, nspec, nsealm, &r); rc != WW_KOKKOS_OK) return rc;
    const ColumnList c(ncol, cols, nsealm, true);
    if (!c.valid) {
      report_line("ww_va_host_wrote_cols refused: a column outside 0..NSEALM or a null list");
      return static_cast<int>(WW_KOKKOS_ERR_BAD_SHAPE);
    }
    return r->wrote_columns(c);
  });
}

int ww_va_host_update(int igrid, float* va, int nspec, int nsealm) {
  return as_status([&]() {
    ResidentVa* r = nullptr;
    if (int rc = bound_va(igrid, va, nspec, nsealm, &r); rc != WW_KOKKOS_OK) return rc;
    return r->host_update();
  });
}

int ww_va_device_zero_cols(int igrid, float* va, int nspec, int nsealm, int ncol,
                           const int* cols) {
  return as_status([&]() {
    ResidentVa* r = nullptr;
    if (int rc = bound_va(igrid, va, nspec, nsealm, &r); rc != WW_KOKKOS_OK) return rc;
    const ColumnList c(ncol, cols, nsealm, false);
    if (!c.valid) {
      report_line("ww_va_device_zero_cols refused: a column outside 0..NSEALM or a null list");
      return static_cast<int>(WW_KOKKOS_ERR_BAD_SHAPE);
    }
    return r->zero_columns(c);
  });
}

int ww_va_device(int igrid, int write) {
  return as_status([&]() {
    auto it = registry().find(igrid);
    if (it == registry().end() || !it->second.bound() || !runtime().ready)
      return static_cast<int>(WW_KOKKOS_ERR_NOT_INITIALISED);
    return it->second.kernel_access(write != 0);
  });
}

void* ww_va_device_ptr(int igrid) {
  auto it = registry().find(igrid);
  return it == registry().end() ? nullptr : static_cast<void*>(it->second.device());
}

int ww_va_state(int igrid) {
  auto it = registry().find(igrid);
  return it == registry().end() || !it->second.bound() ? -1 : static_cast<int>(it->second.state());
}

void ww_va_report(void) {
  const Traffic& t = g_traffic;
  std::fprintf(stderr,
               "ww_b200 [va] traffic: %lld whole uploads (%.2f MB), %lld whole downloads (%.2f MB); "
               "%lld host syncs, %lld kernel syncs\n",
               t.uploads, t.upload_mb, t.downloads, t.download_mb, t.host_syncs, t.kernel_syncs);
  std::fprintf(stderr,
               "ww_b200 [va] columns: %lld partial reads (%lld packed copies, %lld columns), %lld "
               "partial writes (%lld packed copies, %lld columns), %.4f MB packed\n",
               t.col_reads, t.col_read_copies, t.col_read_columns, t.col_writes,
               t.col_write_copies, t.col_write_columns, t.col_mb);
  std::fprintf(stderr,
               "ww_b200 [va] zeroing: %lld host updates, %lld device launches, %lld columns; "
               "%lld audits (WW_KOKKOS_VA_CHECK), %lld poisonings (WW_KOKKOS_VA_POISON)\n",
               t.updates, t.zero_launches, t.zero_columns, t.audits, t.poisonings);
}

}  // extern "C"
