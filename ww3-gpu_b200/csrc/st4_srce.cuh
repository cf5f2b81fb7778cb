// ww3-gpu_b200/csrc/st4_srce.cuh
// Launchers of the ST4 (W3SIN4, W3SDS4, W3SPR4) and W3SRCE kernels (st4_srce_kernel.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

#include "snl1_kernel.cuh"
#include "srce_point.cuh"

namespace wwb {

/// One ST4 grid's scalars and device arrays, as the kernels read them (device-resident copy).
struct St4Dev {
  st4::Params p;
  pt::Fields f;
};

/// Everything a W3SRCE launch reads besides the per-point arrays (device-resident copy).
struct SrceDev {
  srce::Params p;
  pt::SrceGrid g;
  st4::Params q;
  pt::Fields f;
  Snl1Dev n;
  pt::SrceLayout L;
};

/// The flags of one W3SRCE time step.
struct SrceStep {
  int it, inflags24, flogrd57, flogrd58;
  float dtg;
};

/// Threads of every ST4 CTA (one CTA per point).
constexpr int kSt4Block = 256;

/// Threads of a W3SRCE CTA, and the CTAs per SM it is built for: one point's serial chains
/// leave most of its warps waiting at barriers, so more points per SM (their shared part fits
/// four times, their registers four times 128 threads) beat more threads per point.
constexpr int kSrceBlock = pt::kSrceSplit ? 128 : 256;
constexpr int kSrceMinBlocks = pt::kSrceSplit ? 4 : 2;

/// One grid's W3SRCE work buffers: the work queue's counter and the global part of the resident
/// CTAs' working sets (grow-only; it stays in L2 at these sizes). Owned by the grid's context.
struct SrceWork {
  int* counter = nullptr;
  float* scratch = nullptr;
  size_t scratch_n = 0;
  void release() {
    if (counter) cudaFree(counter);
    if (scratch) cudaFree(scratch);
    counter = nullptr;
    scratch = nullptr;
    scratch_n = 0;
  }
};

/// Bytes of dynamic shared memory of the W3SRCE kernel for these tables (the working set of
/// one point); 0 when it exceeds the 227 KiB a CTA can have.
size_t srce_smem_bytes(const pt::SrceLayout& L);

/// W3SDS4 for npts points (arrays as ww_sds4 takes them, device pointers). d is the device copy.
void launch_sds4(const St4Dev* d, const st4::Params& hp, int npts, const float* a, const float* k,
                 const float* cg, const float* ustar, const float* usdir, const float* depth,
                 const float* dair, const float* dlwmean, int f57, int f58, float* srhs,
                 float* ddiag, float* brlambda, float* whitecap, cudaStream_t s);

/// W3SIN4 for npts points (arrays as ww_sin4 takes them, device pointers).
void launch_sin4(const St4Dev* d, const st4::Params& hp, int npts, const float* a,
                 const float* cg, const float* k, const float* u, const float* ustar,
                 const float* drat, const float* as, const float* usdir, const float* z0,
                 float* tauwx, float* tauwy, float* tauwnx, float* tauwny, float* s, float* dd,
                 int* llws, cudaStream_t st);

/// W3SPR4 for npts points; out12 holds the 12 INOUT scalar arrays in ww_spr4's order (ustar,
/// usdir, emean, fmean, fmean1, wnmean, amax, cd, z0, charn, fmeanws, dlwmean), each npts.
void launch_spr4(const St4Dev* d, const st4::Params& hp, int npts, const float* a,
                 const float* cg, const float* wn, const float* u, const float* udir,
                 const float* tauwx, const float* tauwy, const int* llws, float* const* out12,
                 cudaStream_t st);

/// Allocates the work buffers launch_srce needs for npts points of these tables (none when they
/// fit), so that a later launch allocates nothing.
void srce_reserve(const pt::SrceLayout& L, int npts, SrceWork& work, cudaStream_t st);

/// One grid's share of a W3SRCE launch over several grids: its tables (d), step flags, points
/// [first, first + npts) of the launch's work queue and its arrays (as launch_srce takes them).
struct SrceJob {
  const SrceDev* d;
  SrceStep step;
  int npts, first;
  float* spec;
  const int* jsea;
  const float *wn1, *cg1, *pin;
  float *psc, *whitecap, *taubbl, *tauice;
  int* shave;
};

/// A recorded W3SRCE batch: its job (first unset) and working-set layout.
struct SrceRecorded {
  SrceJob job;
  pt::SrceLayout L;
};

/// CTAs per SM of the W3SRCE kernels when every one that fits is resident.
int srce_max_ctas_per_sm(const pt::SrceLayout& L);

/// Limits the W3SRCE kernels to `ctas` CTAs per SM (0: all that fit) with the shared-memory
/// carveout they need, the rest of the SM's memory left to L1 (the autotuner's choice).
void srce_set_ctas_per_sm(const pt::SrceLayout& L, int ctas);

/// CTAs of a W3SRCE launch on npts points of these tables (the resident grid, at most npts).
int srce_resident_ctas(const pt::SrceLayout& L, int npts);

/// Allocates launch_srce_multi's work buffers for `total` points of layout L (synchronous).
void srce_multi_reserve(const pt::SrceLayout& L, int total, SrceWork& work);

/// W3SRCE over several grids' points in one persistent launch with one work queue: jobs_dev
/// (device, njobs entries in order of `first`, total points) all of layout L, work reserved for
/// `total` points (srce_reserve). Launch work only, so it can be captured in a graph.
void launch_srce_multi(const SrceJob* jobs_dev, int njobs, int total, const pt::SrceLayout& L,
                       SrceWork& work, cudaStream_t st);

/// W3SRCE for npts points on a persistent grid whose CTAs take points from a work queue
/// (work.counter, zeroed here), so points with many substeps do not hold up the rest. Point n's
/// spectrum is spec + n * nspec, or, with jsea non-null, the resident VA column
/// spec + jsea[n] * nspec. Per-point packets as ww_srce_batch takes them (device pointers).
void launch_srce(const SrceDev* d, const pt::SrceLayout& L, SrceStep step, int npts,
                 float* spec, const int* jsea, const float* wn1, const float* cg1,
                 const float* pin, float* psc, float* whitecap, float* taubbl, float* tauice,
                 int* shave, SrceWork& work, cudaStream_t st);

}  // namespace wwb
