// ww3-gpu_b200/csrc/snl1_kernel.cu
// W3SNL1 (the DIA) kernels for sm_100a.
//
// Arithmetic: the reference's (ww3-gpu kokkos/src/ww_kokkos/snl1_team.hpp:351-497) operation
// for operation, float32, compiled with -fmad=false and IEEE division, so every output equals
// the CPU reference bit for bit. MAX(a, b) is (a < b) ? b : a as Kokkos::max evaluates it.
//
// Two kernels:
//  * snl1_rowshift_kernel -- the B200 path. A persistent grid of CTAs walks the sea points.
//    Each CTA keeps the point's extended spectrum UE and the eight interaction arrays as
//    (row x NTH) matrices in shared memory and addresses them by the row-shift form of the
//    INSNL1 tables (snl1_tables.hpp): row = IF_m(IFR), column = wrap(ITH + shift_n), computed
//    in registers, so no index table is read in the hot loops. The zero bins (row 0) are
//    written once per CTA; a per-point CON row buffer is double-buffered so a point needs three
//    CTA barriers.
//  * snl1_gather_kernel -- the general form over the 32 index tables, for tables that the
//    row-shift form does not reproduce (e.g. imported tables of another shape).
#include "snl1_kernel.cuh"

#include "libm_dev.cuh"
#include "snl1_tables.hpp"
#include "wwb_common.hpp"

namespace wwb {
namespace {

constexpr float kPi = static_cast<float>(3.141592653589793);
constexpr float kTpiInv = 1.0f / (2.0f * kPi);  // TPIINV of constants.F90 (real.hpp:22-23)

/// Section 1: the depth-scaled proportionality constant CONS (snl1_team.hpp:383-390).
__device__ __forceinline__ float dia_cons(const Snl1Dev& p, float kdmean) {
  const float x0 = p.kdcon * kdmean;
  const float x = (x0 < p.kdmn) ? p.kdmn : x0;
  const float y0 = p.snls3 * x;
  const float x2 = (-1.e15f < y0) ? y0 : -1.e15f;
  return p.snlc1 * (1.0f + p.snls1 / x * (1.0f - p.snls2 * x) * dm::expf(x2));
}

__device__ __forceinline__ int wrapc(int c, int nth) {
  return c < 0 ? c + nth : (c >= nth ? c - nth : c);
}

// ------------------------------------------------------------------------------------------
// Row-shift kernel.
//
// Shared memory (floats): UE rows 0..NFRHGH, then 8 arrays of rows 0..NFRCHG (SA1, SA2, DA1C,
// DA1P, DA1M, DA2C, DA2P, DA2M), then 2 x NK CON (conx) rows, then 8 x NFRCHG ints IF_m rows.
// Slot (row, ith0) of a matrix is row * NTH + ith0; row r >= 1 is frequency IFR = r, row 0 the
// zero bins 1-NTH..0 of the Fortran arrays.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) snl1_rowshift_kernel(
    const Snl1Dev p, const int npts, const float* __restrict__ a, const float* __restrict__ cg,
    const float* __restrict__ kdmean, float* __restrict__ s, float* __restrict__ d) {
  extern __shared__ float smem[];
  const int nth = p.nth, nfr = p.nfr, nfrhgh = p.nfrhgh, nfrchg = p.nfrchg;
  const int nspec = p.nspec, nspecx = p.nspecx, nk = p.nk;
  const int alen = (nfrchg + 1) * nth;
  float* const ue = smem;
  float* const arr = ue + (nfrhgh + 1) * nth;
  float* const conx2 = arr + 8 * alen;
  int* const rows = reinterpret_cast<int*>(conx2 + 2 * nk);
  const int tid = threadIdx.x;

  // Once per CTA: zero rows and the IF_m row maps.
  for (int i = tid; i < nth; i += BLOCK) {
    ue[i] = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k) arr[k * alen + i] = 0.0f;
  }
  for (int i = tid; i < 8 * nfrchg; i += BLOCK) rows[i] = p.ifrow[i];

  // Per-thread column shifts and the stride of the bin loops in (row, column) steps.
  int sh[8];
#pragma unroll
  for (int n = 0; n < 8; ++n) sh[n] = p.shift[n];
  const int dq = BLOCK / nth, dr = BLOCK % nth;
  const int q0 = tid / nth, r0 = tid % nth;
  const float dal1 = p.dal1, dal2 = p.dal2, dal3 = p.dal3;

  int buf = 0;
  for (int ipt = blockIdx.x; ipt < npts; ipt += gridDim.x, buf ^= 1) {
    const float* const ap = a + static_cast<size_t>(ipt) * nspec;
    float* const conx = conx2 + buf * nk;

    // 2a. CON(ISP) = TPIINV / SIG(IFR) * CG(IFR), one value per frequency row.
    for (int k = tid; k < nk; k += BLOCK)
      conx[k] = kTpiInv / __ldg(p.sig + k) * __ldg(cg + static_cast<size_t>(ipt) * nk + k);
    const float cons = dia_cons(p, __ldg(kdmean + ipt));
    __syncthreads();

    // 2b. UE = A / CON over rows 1..NFR; the thread that writes the top row NFR of a column
    //     also marches the parametric tail up that column (snl1_team.hpp:392-426).
    {
      int ifr0 = q0, ith = r0;
      for (int isp = tid; isp < nspec; isp += BLOCK) {
        const float v = __ldcs(ap + isp) / conx[ifr0];
        ue[isp + nth] = v;
        if (ifr0 == nfr - 1) {
          float t = v;
          for (int r = nfr + 1; r <= nfrhgh; ++r) {
            t = t * p.fachfe;
            ue[r * nth + ith] = t;
          }
        }
        ith += dr;
        ifr0 += dq;
        if (ith >= nth) {
          ith -= nth;
          ++ifr0;
        }
      }
    }
    __syncthreads();

    // 3. Interactions over the extended spectrum (snl1_team.hpp:433-473).
    {
      int ifr0 = q0, ith = r0;
      for (int isp = tid; isp < nspecx; isp += BLOCK) {
        int c[8];
#pragma unroll
        for (int n = 0; n < 8; ++n) c[n] = wrapc(ith + sh[n], nth);
        const int r1 = rows[0 * nfrchg + ifr0] * nth;  // IF1
        const int r2 = rows[1 * nfrchg + ifr0] * nth;  // IF2
        const int r3 = rows[2 * nfrchg + ifr0] * nth;  // IF3
        const int r4 = rows[3 * nfrchg + ifr0] * nth;  // IF4
        const float e00 = ue[isp + nth];
        // IP11..IP14 = (IT2,IF2) (IT1,IF2) (IT2,IF1) (IT1,IF1); IM1j = (IT8|IT7, IF4|IF3);
        // IP2j = (IT6|IT5, IF2|IF1); IM2j = (IT4|IT3, IF4|IF3).
        const float ep1 = p.awg[0] * ue[r2 + c[1]] + p.awg[1] * ue[r2 + c[0]] +
                          p.awg[2] * ue[r1 + c[1]] + p.awg[3] * ue[r1 + c[0]];
        const float em1 = p.awg[4] * ue[r4 + c[7]] + p.awg[5] * ue[r4 + c[6]] +
                          p.awg[6] * ue[r3 + c[7]] + p.awg[7] * ue[r3 + c[6]];
        const float ep2 = p.awg[0] * ue[r2 + c[5]] + p.awg[1] * ue[r2 + c[4]] +
                          p.awg[2] * ue[r1 + c[5]] + p.awg[3] * ue[r1 + c[4]];
        const float em2 = p.awg[4] * ue[r4 + c[3]] + p.awg[5] * ue[r4 + c[2]] +
                          p.awg[6] * ue[r3 + c[3]] + p.awg[7] * ue[r3 + c[2]];
        const float ca = cons * p.af11_row[ifr0];
        const float factor = ca * e00;
        const float sa1a = e00 * (ep1 * dal1 + em1 * dal2);
        const float sa1b = sa1a - ep1 * em1 * dal3;
        const float sa2a = e00 * (ep2 * dal1 + em2 * dal2);
        const float sa2b = sa2a - ep2 * em2 * dal3;
        const int o = isp + nth;
        arr[0 * alen + o] = factor * sa1b;
        arr[1 * alen + o] = factor * sa2b;
        arr[2 * alen + o] = ca * (sa1a + sa1b);
        arr[3 * alen + o] = factor * (dal1 * e00 - dal3 * em1);
        arr[4 * alen + o] = factor * (dal2 * e00 - dal3 * ep1);
        arr[5 * alen + o] = ca * (sa2a + sa2b);
        arr[6 * alen + o] = factor * (dal1 * e00 - dal3 * em2);
        arr[7 * alen + o] = factor * (dal2 * e00 - dal3 * ep2);
        ith += dr;
        ifr0 += dq;
        if (ith >= nth) {
          ith -= nth;
          ++ifr0;
        }
      }
    }
    __syncthreads();

    // 4. Source and diagonal terms (snl1_team.hpp:475-496).
    {
      const float* const sa1 = arr;
      const float* const sa2 = arr + alen;
      const float* const da1c = arr + 2 * alen;
      const float* const da1p = arr + 3 * alen;
      const float* const da1m = arr + 4 * alen;
      const float* const da2c = arr + 5 * alen;
      const float* const da2p = arr + 6 * alen;
      const float* const da2m = arr + 7 * alen;
      float* const sp = s + static_cast<size_t>(ipt) * nspec;
      float* const dp = d + static_cast<size_t>(ipt) * nspec;
      int ifr0 = q0, ith = r0;
      for (int isp = tid; isp < nspec; isp += BLOCK) {
        int c[8];
#pragma unroll
        for (int n = 0; n < 8; ++n) c[n] = wrapc(ith + sh[n], nth);
        const int r5 = rows[4 * nfrchg + ifr0] * nth;  // IF5
        const int r6 = rows[5 * nfrchg + ifr0] * nth;  // IF6
        const int r7 = rows[6 * nfrchg + ifr0] * nth;  // IF7
        const int r8 = rows[7 * nfrchg + ifr0] * nth;  // IF8
        const int o = isp + nth;
        // IC11..IC81 = (IT6,IF6) (IT5,IF6) (IT6,IF5) (IT5,IF5) (IT4,IF8) (IT3,IF8) (IT4,IF7)
        // (IT3,IF7); IC12..IC82 = (IT2,IF6) (IT1,IF6) (IT2,IF5) (IT1,IF5) (IT8,IF8) (IT7,IF8)
        // (IT8,IF7) (IT7,IF7).
        const float sv = conx[ifr0] * (-2.0f * (sa1[o] + sa2[o]) +
                                       p.awg[0] * (sa1[r6 + c[5]] + sa2[r6 + c[1]]) +
                                       p.awg[1] * (sa1[r6 + c[4]] + sa2[r6 + c[0]]) +
                                       p.awg[2] * (sa1[r5 + c[5]] + sa2[r5 + c[1]]) +
                                       p.awg[3] * (sa1[r5 + c[4]] + sa2[r5 + c[0]]) +
                                       p.awg[4] * (sa1[r8 + c[3]] + sa2[r8 + c[7]]) +
                                       p.awg[5] * (sa1[r8 + c[2]] + sa2[r8 + c[6]]) +
                                       p.awg[6] * (sa1[r7 + c[3]] + sa2[r7 + c[7]]) +
                                       p.awg[7] * (sa1[r7 + c[2]] + sa2[r7 + c[6]]));
        const float dv = -2.0f * (da1c[o] + da2c[o]) +
                         p.swg[0] * (da1p[r6 + c[5]] + da2p[r6 + c[1]]) +
                         p.swg[1] * (da1p[r6 + c[4]] + da2p[r6 + c[0]]) +
                         p.swg[2] * (da1p[r5 + c[5]] + da2p[r5 + c[1]]) +
                         p.swg[3] * (da1p[r5 + c[4]] + da2p[r5 + c[0]]) +
                         p.swg[4] * (da1m[r8 + c[3]] + da2m[r8 + c[7]]) +
                         p.swg[5] * (da1m[r8 + c[2]] + da2m[r8 + c[6]]) +
                         p.swg[6] * (da1m[r7 + c[3]] + da2m[r7 + c[7]]) +
                         p.swg[7] * (da1m[r7 + c[2]] + da2m[r7 + c[6]]);
        __stcs(sp + isp, sv);
        __stcs(dp + isp, dv);
        ith += dr;
        ifr0 += dq;
        if (ith >= nth) {
          ith -= nth;
          ++ifr0;
        }
      }
    }
    // No barrier here: the next point writes the other CON buffer, and UE / the interaction
    // arrays only after the CON barrier, which every thread reaches after its section 4.
  }
}

// ------------------------------------------------------------------------------------------
// Gather kernel: one CTA per point over the index tables (general form). Shared memory:
// UE (NSPECY + NTH), 8 x (NSPECX + NTH), CON per row (NK).
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) snl1_gather_kernel(
    const Snl1Dev p, const int npts, const float* __restrict__ a, const float* __restrict__ cg,
    const float* __restrict__ kdmean, float* __restrict__ s, float* __restrict__ d) {
  extern __shared__ float smem[];
  const int nth = p.nth, nfr = p.nfr, nfrhgh = p.nfrhgh, nspec = p.nspec, nspecx = p.nspecx;
  const int xl = nspecx + nth;
  float* const ue = smem;
  float* const sa1 = ue + (p.nfrhgh * nth + nth);
  float* const sa2 = sa1 + xl;
  float* const da1c = sa2 + xl;
  float* const da1p = da1c + xl;
  float* const da1m = da1p + xl;
  float* const da2c = da1m + xl;
  float* const da2p = da2c + xl;
  float* const da2m = da2p + xl;
  float* const conx = da2m + xl;
  const int tid = threadIdx.x;
  const int ipt = blockIdx.x;
  if (ipt >= npts) return;
  const float* const ap = a + static_cast<size_t>(ipt) * nspec;

  for (int k = tid; k < p.nk; k += BLOCK)
    conx[k] = kTpiInv / p.sig[k] * cg[static_cast<size_t>(ipt) * p.nk + k];
  for (int i = tid; i < nth; i += BLOCK) {
    ue[i] = sa1[i] = sa2[i] = da1c[i] = da1p[i] = da1m[i] = 0.0f;
    da2c[i] = da2p[i] = da2m[i] = 0.0f;
  }
  const float cons = dia_cons(p, kdmean[ipt]);
  __syncthreads();
  for (int isp = tid; isp < nspec; isp += BLOCK) ue[isp + nth] = ap[isp] / conx[isp / nth];
  __syncthreads();
  for (int ifr = nfr; ifr < nfrhgh; ++ifr) {
    for (int ith = tid; ith < nth; ith += BLOCK) {
      const int isp = ith + ifr * nth;
      ue[isp + nth] = ue[isp] * p.fachfe;
    }
    __syncthreads();
  }
  const int* const T = p.ipim;
  for (int isp = tid; isp < nspecx; isp += BLOCK) {
#define U(j) ue[__ldg(T + (j) * nspecx + isp) + nth]
    const float e00 = ue[isp + nth];
    const float ep1 = p.awg[0] * U(0) + p.awg[1] * U(1) + p.awg[2] * U(2) + p.awg[3] * U(3);
    const float em1 = p.awg[4] * U(4) + p.awg[5] * U(5) + p.awg[6] * U(6) + p.awg[7] * U(7);
    const float ep2 = p.awg[0] * U(8) + p.awg[1] * U(9) + p.awg[2] * U(10) + p.awg[3] * U(11);
    const float em2 = p.awg[4] * U(12) + p.awg[5] * U(13) + p.awg[6] * U(14) + p.awg[7] * U(15);
#undef U
    const float ca = cons * __ldg(p.af11 + isp);
    const float factor = ca * e00;
    const float sa1a = e00 * (ep1 * p.dal1 + em1 * p.dal2);
    const float sa1b = sa1a - ep1 * em1 * p.dal3;
    const float sa2a = e00 * (ep2 * p.dal1 + em2 * p.dal2);
    const float sa2b = sa2a - ep2 * em2 * p.dal3;
    sa1[isp + nth] = factor * sa1b;
    sa2[isp + nth] = factor * sa2b;
    da1c[isp + nth] = ca * (sa1a + sa1b);
    da1p[isp + nth] = factor * (p.dal1 * e00 - p.dal3 * em1);
    da1m[isp + nth] = factor * (p.dal2 * e00 - p.dal3 * ep1);
    da2c[isp + nth] = ca * (sa2a + sa2b);
    da2p[isp + nth] = factor * (p.dal1 * e00 - p.dal3 * em2);
    da2m[isp + nth] = factor * (p.dal2 * e00 - p.dal3 * ep2);
  }
  __syncthreads();
  const int* const C = p.ic;
  for (int isp = tid; isp < nspec; isp += BLOCK) {
#define C1(j) (__ldg(C + (j) * nspec + isp) + nth)
#define C2(j) (__ldg(C + (8 + (j)) * nspec + isp) + nth)
    const float sv =
        conx[isp / nth] *
        (-2.0f * (sa1[isp + nth] + sa2[isp + nth]) + p.awg[0] * (sa1[C1(0)] + sa2[C2(0)]) +
         p.awg[1] * (sa1[C1(1)] + sa2[C2(1)]) + p.awg[2] * (sa1[C1(2)] + sa2[C2(2)]) +
         p.awg[3] * (sa1[C1(3)] + sa2[C2(3)]) + p.awg[4] * (sa1[C1(4)] + sa2[C2(4)]) +
         p.awg[5] * (sa1[C1(5)] + sa2[C2(5)]) + p.awg[6] * (sa1[C1(6)] + sa2[C2(6)]) +
         p.awg[7] * (sa1[C1(7)] + sa2[C2(7)]));
    const float dv = -2.0f * (da1c[isp + nth] + da2c[isp + nth]) +
                     p.swg[0] * (da1p[C1(0)] + da2p[C2(0)]) + p.swg[1] * (da1p[C1(1)] + da2p[C2(1)]) +
                     p.swg[2] * (da1p[C1(2)] + da2p[C2(2)]) + p.swg[3] * (da1p[C1(3)] + da2p[C2(3)]) +
                     p.swg[4] * (da1m[C1(4)] + da2m[C2(4)]) + p.swg[5] * (da1m[C1(5)] + da2m[C2(5)]) +
                     p.swg[6] * (da1m[C1(6)] + da2m[C2(6)]) + p.swg[7] * (da1m[C1(7)] + da2m[C2(7)]);
#undef C1
#undef C2
    s[static_cast<size_t>(ipt) * nspec + isp] = sv;
    d[static_cast<size_t>(ipt) * nspec + isp] = dv;
  }
}

constexpr int kRowShiftBlock = 288;
constexpr int kGatherBlock = 256;

int g_rowshift_ctas_per_sm = -1;  // occupancy, per device size (computed on first launch)
size_t g_rowshift_smem_cached = 0;

}  // namespace

size_t snl1_gather_smem(const Snl1Dev& p) {
  return sizeof(float) * (static_cast<size_t>(p.nfrhgh + 1) * p.nth +
                          8 * static_cast<size_t>(p.nspecx + p.nth) + p.nk);
}

size_t snl1_rowshift_smem(const Snl1Dev& p) {
  return sizeof(float) * (static_cast<size_t>(p.nfrhgh + 1) * p.nth +
                          8 * static_cast<size_t>(p.nfrchg + 1) * p.nth + 2 * p.nk) +
         sizeof(int) * 8 * static_cast<size_t>(p.nfrchg);
}

void launch_snl1(int kernel, const Snl1Dev& p, int npts, const float* a, const float* cg,
                 const float* kdmean, float* s, float* d, cudaStream_t stream) {
  if (npts <= 0) return;
  if (kernel == kSnl1RowShift) {
    const size_t smem = snl1_rowshift_smem(p);
    auto k = snl1_rowshift_kernel<kRowShiftBlock>;
    if (g_rowshift_ctas_per_sm < 0 || g_rowshift_smem_cached != smem) {
      WWB_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(smem)));
      int per_sm = 0;
      WWB_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kRowShiftBlock, smem));
      if (per_sm < 1) throw CudaError(cudaErrorInvalidConfiguration, "snl1 row-shift occupancy");
      g_rowshift_ctas_per_sm = per_sm;
      g_rowshift_smem_cached = smem;
    }
    const long long resident =
        static_cast<long long>(g_rowshift_ctas_per_sm) * runtime().sm_count;
    const int grid = static_cast<int>(npts < resident ? npts : resident);
    k<<<grid, kRowShiftBlock, smem, stream>>>(p, npts, a, cg, kdmean, s, d);
    WWB_CHECK(cudaGetLastError());
  } else {
    const size_t smem = snl1_gather_smem(p);
    auto k = snl1_gather_kernel<kGatherBlock>;
    WWB_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(smem)));
    k<<<npts, kGatherBlock, smem, stream>>>(p, npts, a, cg, kdmean, s, d);
    WWB_CHECK(cudaGetLastError());
  }
}

}  // namespace wwb
