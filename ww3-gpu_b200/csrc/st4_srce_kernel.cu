// ww3-gpu_b200/csrc/st4_srce_kernel.cu
// The ST4 source terms and W3SRCE on sm_100a: one CTA of 256 threads per sea point, the point's
// working set in shared memory, the phases of st4_point.cuh / srce_point.cuh.
//
// W3SRCE runs on a persistent grid: each CTA takes the next point from a global counter as it
// finishes one, so the uneven number of substeps per point (the dynamic integration stops when
// the point's DTTOT reaches DTG) balances across the SMs instead of leaving a tail of idle CTAs.
// The scalar state of a point sits in static shared memory, its spectra and work arrays in
// dynamic shared memory (about 100 KiB at 36x36, two CTAs per SM).
#include "st4_srce.cuh"

#include "wwb_common.hpp"

namespace wwb {
namespace {

__global__ void __launch_bounds__(kSt4Block) sds4_kernel(
    const St4Dev* __restrict__ d, int npts, const float* a, const float* k, const float* cg,
    const float* ustar, const float* usdir, const float* depth, const float* dair,
    const float* dlwmean, int f57, int f58, float* srhs, float* ddiag, float* brlambda,
    float* whitecap) {
  extern __shared__ __align__(16) float smem[];
  __shared__ pt::Sds4Sh sh;
  const st4::Params& p = d->p;
  const pt::Cta cta{static_cast<int>(threadIdx.x), static_cast<int>(blockDim.x)};
  float* const w = smem;
  float* const w2 = w + ((pt::sds4_work_reals(p) + 3) & ~3);
  int* const iw = reinterpret_cast<int*>(w2 + pt::sds4_work2_reals(p));
  for (int n = blockIdx.x; n < npts; n += gridDim.x) {
    const size_t os = static_cast<size_t>(n) * p.nspec, ok = static_cast<size_t>(n) * p.nk;
    pt::sds4(cta, p, d->f, a + os, k + ok, cg + ok, ustar[n], usdir[n], depth[n], dair[n],
             dlwmean[n], f57, f58, srhs + os, ddiag + os, brlambda + os,
             whitecap + 4 * static_cast<size_t>(n), w, w2, iw, sh);
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kSt4Block) sin4_kernel(
    const St4Dev* __restrict__ d, int npts, const float* a, const float* cg, const float* k,
    const float* u, const float* ustar, const float* drat, const float* as, const float* usdir,
    const float* z0, float* tauwx, float* tauwy, float* tauwnx, float* tauwny, float* s,
    float* dd, int* llws) {
  extern __shared__ __align__(16) float smem[];
  __shared__ pt::Sin4Sh sh;
  const st4::Params& p = d->p;
  const pt::Cta cta{static_cast<int>(threadIdx.x), static_cast<int>(blockDim.x)};
  float* const dstab = smem;
  float* const eb = dstab + 3 * p.nspec;
  for (int n = blockIdx.x; n < npts; n += gridDim.x) {
    const size_t os = static_cast<size_t>(n) * p.nspec, ok = static_cast<size_t>(n) * p.nk;
    pt::sin4(cta, p, d->f, a + os, cg + ok, k + os, p.nth, u[n], ustar[n], drat[n], as[n],
             usdir[n], z0[n], tauwx + n, tauwy + n, tauwnx + n, tauwny + n, s + os, dd + os,
             llws + os, dstab, eb, sh);
    __syncthreads();
  }
}

struct Spr4Ptrs {
  float* o[12];
};

__global__ void __launch_bounds__(kSt4Block) spr4_kernel(
    const St4Dev* __restrict__ d, int npts, const float* a, const float* cg, const float* wn,
    const float* u, const float* udir, const float* tauwx, const float* tauwy, const int* llws,
    Spr4Ptrs out) {
  extern __shared__ __align__(16) float smem[];
  __shared__ pt::Spr4Out o;
  const st4::Params& p = d->p;
  const pt::Cta cta{static_cast<int>(threadIdx.x), static_cast<int>(blockDim.x)};
  for (int n = blockIdx.x; n < npts; n += gridDim.x) {
    const size_t os = static_cast<size_t>(n) * p.nspec, ok = static_cast<size_t>(n) * p.nk;
    if (threadIdx.x == 0) {
      float* const f = &o.ustar;
      for (int j = 0; j < 12; ++j) f[j] = out.o[j][n];
    }
    __syncthreads();
    pt::spr4(cta, p, d->f, a + os, cg + ok, wn + ok, u[n], udir[n], tauwx[n], tauwy[n],
             llws + os, o, smem, smem + ((pt::spr4_work_reals(p) + 3) & ~3));
    if (threadIdx.x == 0) {
      const float* const f = &o.ustar;
      for (int j = 0; j < 12; ++j) out.o[j][n] = f[j];
    }
    __syncthreads();
  }
}

/// One sea point of a W3SRCE batch by the whole CTA: its spectrum (VA column jsea[n], or row n)
/// and packets into the working set, srce_point, and back. w is the CTA's dynamic shared
/// memory, gw its slice of the global scratch.
__device__ __forceinline__ void srce_one(const SrceDev* __restrict__ d, const SrceStep& step,
                                         int n, float* spec, const int* jsea, const float* wn1,
                                         const float* cg1, const float* pin, float* psc,
                                         float* whitecap, float* taubbl, float* tauice,
                                         int* shave, float* w, float* gw, pt::SrceSh& sh) {
  const pt::SrceLayout& L = d->L;
  const int ns = L.nspec, nk = L.nk;
  const pt::Cta cta{static_cast<int>(threadIdx.x), static_cast<int>(blockDim.x)};
  float* const sp = spec + (jsea ? static_cast<size_t>(jsea[n]) : static_cast<size_t>(n)) * ns;
  for (int i = threadIdx.x; i < ns; i += blockDim.x) w[L.spec + i] = sp[i];
  for (int i = threadIdx.x; i < nk; i += blockDim.x) {
    w[L.wn1 + i] = wn1[static_cast<size_t>(n) * nk + i];
    w[L.cg1 + i] = cg1[static_cast<size_t>(n) * nk + i];
  }
  if (threadIdx.x == 0)
    pt::srce_psc_in(sh, psc + static_cast<size_t>(n) * srce::NPSC,
                    whitecap + 4 * static_cast<size_t>(n), taubbl + 2 * static_cast<size_t>(n),
                    tauice + 2 * static_cast<size_t>(n));
  __syncthreads();
  const pt::SrceCtx x{&d->p, &d->g, &d->q, &d->f, &d->n,
                      pt::srce_in(step.it, step.inflags24, step.flogrd57, step.flogrd58, step.dtg,
                                  pin + static_cast<size_t>(n) * srce::NPIN),
                      w, gw, &L, &sh};
  pt::srce_point(cta, x);
  for (int i = threadIdx.x; i < ns; i += blockDim.x) sp[i] = w[L.spec + i];
  if (threadIdx.x == 0)
    pt::srce_psc_out(sh, psc + static_cast<size_t>(n) * srce::NPSC,
                     whitecap + 4 * static_cast<size_t>(n), taubbl + 2 * static_cast<size_t>(n),
                     tauice + 2 * static_cast<size_t>(n), shave + n);
  __syncthreads();
}

__global__ void __launch_bounds__(kSrceBlock, kSrceMinBlocks) srce_kernel(
    const SrceDev* __restrict__ d, SrceStep step, int npts, float* spec, const int* jsea,
    const float* wn1, const float* cg1, const float* pin, float* psc, float* whitecap,
    float* taubbl, float* tauice, int* shave, int* counter, float* scratch) {
  extern __shared__ __align__(16) float w[];
  __shared__ pt::SrceSh sh;
  __shared__ int cur;
  float* const gw = scratch + static_cast<size_t>(blockIdx.x) * static_cast<size_t>(d->L.total_g);
  for (;;) {
    if (threadIdx.x == 0) cur = atomicAdd(counter, 1);
    __syncthreads();
    const int n = cur;
    if (n >= npts) break;
    srce_one(d, step, n, spec, jsea, wn1, cg1, pin, psc, whitecap, taubbl, tauice, shave, w, gw,
             sh);
  }
}

/// W3SRCE over the points of several grids in one persistent launch: one work queue over
/// (grid, point), the job of queue entry q the last one whose first entry is <= q. Every job has
/// the same working-set layout (checked on the host), so one CTA takes any grid's points.
__global__ void __launch_bounds__(kSrceBlock, kSrceMinBlocks) srce_multi_kernel(
    const SrceJob* __restrict__ jobs, int njobs, int total, int* counter, float* scratch) {
  extern __shared__ __align__(16) float w[];
  __shared__ pt::SrceSh sh;
  __shared__ int cur;
  float* const gw =
      scratch + static_cast<size_t>(blockIdx.x) * static_cast<size_t>(jobs[0].d->L.total_g);
  for (;;) {
    if (threadIdx.x == 0) cur = atomicAdd(counter, 1);
    __syncthreads();
    const int q = cur;
    if (q >= total) break;
    int lo = 0, hi = njobs - 1;  // the job holding q: first[lo] <= q < first[lo + 1]
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (jobs[mid].first <= q) lo = mid;
      else hi = mid - 1;
    }
    const SrceJob& j = jobs[lo];
    srce_one(j.d, j.step, q - j.first, j.spec, j.jsea, j.wn1, j.cg1, j.pin, j.psc, j.whitecap,
             j.taubbl, j.tauice, j.shave, w, gw, sh);
  }
}

/// CTAs per SM of the W3SRCE kernels (0: all that fit), set by the autotuner.
int g_srce_ctas_per_sm = 0;

/// Resident CTAs per SM of a kernel at this shared memory, at least 1 (for the W3SRCE kernels,
/// at most the autotuner's choice).
template <class K>
int resident_grid(K k, size_t smem, int npts, int block = kSt4Block, bool srce = false) {
  WWB_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem)));
  int per_sm = 0;
  WWB_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, block, smem));
  if (per_sm < 1) throw CudaError(cudaErrorInvalidConfiguration, "st4/srce occupancy");
  if (srce && g_srce_ctas_per_sm > 0 && g_srce_ctas_per_sm < per_sm)
    per_sm = g_srce_ctas_per_sm;
  const long long resident = static_cast<long long>(per_sm) * runtime().sm_count;
  return static_cast<int>(npts < resident ? npts : resident);
}

}  // namespace

int srce_max_ctas_per_sm(const pt::SrceLayout& L) {
  const size_t smem = srce_smem_bytes(L);
  if (smem == 0) throw CudaError(cudaErrorInvalidConfiguration, "W3SRCE working set too large");
  const int keep = g_srce_ctas_per_sm;
  g_srce_ctas_per_sm = 0;
  WWB_CHECK(cudaFuncSetAttribute(srce_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutDefault));
  const int all = resident_grid(srce_kernel, smem, 1 << 30, kSrceBlock, true) / runtime().sm_count;
  srce_set_ctas_per_sm(L, keep);  // the carveout of the current choice again
  return all;
}

void srce_set_ctas_per_sm(const pt::SrceLayout& L, int ctas) {
  const size_t smem = srce_smem_bytes(L);
  if (smem == 0) throw CudaError(cudaErrorInvalidConfiguration, "W3SRCE working set too large");
  g_srce_ctas_per_sm = ctas > 0 ? ctas : 0;
  // The shared-memory carveout just large enough for that many CTAs (their dynamic and static
  // shared memory and the 1 KiB the system keeps per CTA): the rest of the SM's 256 KiB is L1.
  int pct = cudaSharedmemCarveoutDefault;
  if (ctas > 0) {
    const size_t per_cta = smem + sizeof(pt::SrceSh) + 16 + 1024;
    pct = static_cast<int>((100 * ctas * per_cta + 228 * 1024 - 1) / (228 * 1024));
    if (pct > 100) pct = 100;
  }
  WWB_CHECK(cudaFuncSetAttribute(srce_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
  WWB_CHECK(
      cudaFuncSetAttribute(srce_multi_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
}

size_t srce_smem_bytes(const pt::SrceLayout& L) {
  const size_t b = static_cast<size_t>(L.total_s) * sizeof(float) + 16;
  return b + sizeof(pt::SrceSh) <= 227 * 1024 ? b : 0;
}

void launch_sds4(const St4Dev* d, const st4::Params& hp, int npts, const float* a, const float* k,
                 const float* cg, const float* ustar, const float* usdir, const float* depth,
                 const float* dair, const float* dlwmean, int f57, int f58, float* srhs,
                 float* ddiag, float* brlambda, float* whitecap, cudaStream_t s) {
  if (npts <= 0) return;
  const size_t smem = sizeof(float) * (((pt::sds4_work_reals(hp) + 3) & ~3) +
                                       pt::sds4_work2_reals(hp) + pt::sds4_work_ints(hp));
  const int grid = resident_grid(sds4_kernel, smem, npts);
  sds4_kernel<<<grid, kSt4Block, smem, s>>>(d, npts, a, k, cg, ustar, usdir, depth, dair, dlwmean,
                                            f57, f58, srhs, ddiag, brlambda, whitecap);
  WWB_CHECK(cudaGetLastError());
}

void launch_sin4(const St4Dev* d, const st4::Params& hp, int npts, const float* a,
                 const float* cg, const float* k, const float* u, const float* ustar,
                 const float* drat, const float* as, const float* usdir, const float* z0,
                 float* tauwx, float* tauwy, float* tauwnx, float* tauwny, float* s, float* dd,
                 int* llws, cudaStream_t st) {
  if (npts <= 0) return;
  const size_t smem = sizeof(float) * (3 * static_cast<size_t>(hp.nspec) + pt::sin4_nk_work(hp));
  const int grid = resident_grid(sin4_kernel, smem, npts);
  sin4_kernel<<<grid, kSt4Block, smem, st>>>(d, npts, a, cg, k, u, ustar, drat, as, usdir, z0,
                                             tauwx, tauwy, tauwnx, tauwny, s, dd, llws);
  WWB_CHECK(cudaGetLastError());
}

void launch_spr4(const St4Dev* d, const st4::Params& hp, int npts, const float* a,
                 const float* cg, const float* wn, const float* u, const float* udir,
                 const float* tauwx, const float* tauwy, const int* llws, float* const* out12,
                 cudaStream_t st) {
  if (npts <= 0) return;
  Spr4Ptrs o;
  for (int j = 0; j < 12; ++j) o.o[j] = out12[j];
  const size_t smem = sizeof(float) * (((pt::spr4_work_reals(hp) + 3) & ~3) +
                                       static_cast<size_t>(pt::spr4_terms_reals(hp)));
  const int grid = resident_grid(spr4_kernel, smem, npts);
  spr4_kernel<<<grid, kSt4Block, smem, st>>>(d, npts, a, cg, wn, u, udir, tauwx, tauwy, llws, o);
  WWB_CHECK(cudaGetLastError());
}

void srce_reserve(const pt::SrceLayout& L, int npts, SrceWork& work, cudaStream_t st) {
  if (npts <= 0) return;
  const size_t smem = srce_smem_bytes(L);
  if (smem == 0) throw CudaError(cudaErrorInvalidConfiguration, "W3SRCE working set too large");
  const int grid = resident_grid(srce_kernel, smem, npts, kSrceBlock, true);
  const size_t need = static_cast<size_t>(grid) * static_cast<size_t>(L.total_g);
  if (work.counter == nullptr) WWB_CHECK(cudaMalloc(&work.counter, sizeof(int)));
  if (need > work.scratch_n) {
    WWB_CHECK(cudaStreamSynchronize(st));
    if (work.scratch) WWB_CHECK(cudaFree(work.scratch));
    work.scratch = nullptr;
    work.scratch_n = 0;
    WWB_CHECK(cudaMalloc(&work.scratch, need * sizeof(float)));
    work.scratch_n = need;
  }
}

int srce_resident_ctas(const pt::SrceLayout& L, int npts) {
  const size_t smem = srce_smem_bytes(L);
  if (smem == 0) throw CudaError(cudaErrorInvalidConfiguration, "W3SRCE working set too large");
  return resident_grid(srce_kernel, smem, npts, kSrceBlock, true);
}

void srce_multi_reserve(const pt::SrceLayout& L, int total, SrceWork& work) {
  const size_t smem = srce_smem_bytes(L);
  if (smem == 0) throw CudaError(cudaErrorInvalidConfiguration, "W3SRCE working set too large");
  const int grid = resident_grid(srce_multi_kernel, smem, total > 0 ? total : 1, kSrceBlock, true);
  const size_t need = static_cast<size_t>(grid) * static_cast<size_t>(L.total_g);
  if (work.counter == nullptr) WWB_CHECK(cudaMalloc(&work.counter, sizeof(int)));
  if (need > work.scratch_n) {
    if (work.scratch) WWB_CHECK(cudaFree(work.scratch));
    work.scratch = nullptr;
    work.scratch_n = 0;
    WWB_CHECK(cudaMalloc(&work.scratch, need * sizeof(float)));
    work.scratch_n = need;
  }
}

void launch_srce_multi(const SrceJob* jobs_dev, int njobs, int total, const pt::SrceLayout& L,
                       SrceWork& work, cudaStream_t st) {
  if (total <= 0) return;
  const size_t smem = srce_smem_bytes(L);
  if (smem == 0) throw CudaError(cudaErrorInvalidConfiguration, "W3SRCE working set too large");
  const int grid = resident_grid(srce_multi_kernel, smem, total, kSrceBlock, true);
  if (work.counter == nullptr ||
      static_cast<size_t>(grid) * static_cast<size_t>(L.total_g) > work.scratch_n)
    throw CudaError(cudaErrorInvalidValue, "launch_srce_multi: work buffers not reserved");
  WWB_CHECK(cudaMemsetAsync(work.counter, 0, sizeof(int), st));
  srce_multi_kernel<<<grid, kSrceBlock, smem, st>>>(jobs_dev, njobs, total, work.counter,
                                                    work.scratch);
  WWB_CHECK(cudaGetLastError());
}

void launch_srce(const SrceDev* d, const pt::SrceLayout& L, SrceStep step, int npts,
                 float* spec, const int* jsea, const float* wn1, const float* cg1,
                 const float* pin, float* psc, float* whitecap, float* taubbl, float* tauice,
                 int* shave, SrceWork& work, cudaStream_t st) {
  if (npts <= 0) return;
  const size_t smem = srce_smem_bytes(L);
  if (smem == 0) throw CudaError(cudaErrorInvalidConfiguration, "W3SRCE working set too large");
  const int grid = resident_grid(srce_kernel, smem, npts, kSrceBlock, true);
  // The work buffers fit after srce_reserve; otherwise (re)allocate them first, after the
  // previous launches on this stream that may still read the old ones.
  srce_reserve(L, npts, work, st);
  WWB_CHECK(cudaMemsetAsync(work.counter, 0, sizeof(int), st));
  srce_kernel<<<grid, kSrceBlock, smem, st>>>(d, step, npts, spec, jsea, wn1, cg1, pin, psc,
                                              whitecap, taubbl, tauice, shave, work.counter,
                                              work.scratch);
  WWB_CHECK(cudaGetLastError());
}

}  // namespace wwb
