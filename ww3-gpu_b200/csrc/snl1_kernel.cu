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

// ------------------------------------------------------------------------------------------
// Band kernel: the B200 path.
//
// Persistent CTAs walk the sea points. Thread t owns direction column ITH = t % NTH and a band
// of BR consecutive frequency rows (band t / NTH), the same band in sections 3 and 4. Along its
// band it slides register windows over the rows the quadruplet reads: the IF1/IF2 rows (the
// "plus" pair) and the IF3/IF4 rows (the "minus" pair) in section 3, the IF5/IF6 and IF7/IF8
// rows in section 4, each window holding the four wrapped columns of that pair, so moving one
// row up loads one new row of each pair. The eight wrapped columns are computed once per
// thread. DA1C and DA2C are read back only at their own bin, so their sum is kept instead of
// the two arrays: six interaction arrays and one sum array live in shared memory. The next point's A and CG are brought
// into a shared staging buffer by one TMA bulk copy (cp.async.bulk, completed on an mbarrier)
// while the current point is computed. Every floating-point operation is the reference's, in
// its order (snl1_team.hpp:383-496).
//
// Row algebra (INSNL1 section 7): IF1 = f + IFRP, IF2 = IF1 + 1, IF3 = max(0, f + IFRM),
// IF4 = max(0, f + IFRM - 1), IF5 = max(0, f - IFRP), IF6 = max(0, f - IFRP - 1),
// IF7 = f - IFRM, IF8 = IF7 + 1, with IFRP >= 0 >= IFRM.
//
// Shared memory (floats): UE rows 0..NFRHGH; SA1, SA2, DA1P, DA1M, DA2P, DA2M rows 0..NFRCHG;
// DC = DA1C + DA2C over the NSPEC bins (read back only by the thread that wrote it); CON rows
// (2 x NK, double-buffered by point parity); AF11 rows (NFRCHG); the staging buffer
// (NSPEC + NK, 16-byte aligned); the mbarrier.

constexpr unsigned kWaitLimit = 1u << 22;  // bounded mbarrier waits (about a second)

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

/// One elected thread: expect `bytes` and start the bulk copies of A and CG of point `ipt`.
__device__ __forceinline__ void tma_fetch_point(uint64_t* bar, float* stage, const float* a,
                                                const float* cg, int ipt, int nspec, int nk) {
  const unsigned bytes_a = static_cast<unsigned>(nspec) * 4u;
  const unsigned bytes_c = static_cast<unsigned>(nk) * 4u;
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes_a + bytes_c)
               : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(stage)),
      "l"(a + static_cast<size_t>(ipt) * nspec), "r"(bytes_a), "r"(smem_u32(bar))
      : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(stage + nspec)),
      "l"(cg + static_cast<size_t>(ipt) * nk), "r"(bytes_c), "r"(smem_u32(bar))
      : "memory");
}

/// Wait for phase `parity` of the mbarrier, giving up after kWaitLimit polls: then the status
/// word records it (the host reports the failure) and false is returned, and the caller's CTA
/// stops at its next barrier (see the point loops) without starting another bulk copy.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, int* err) {
  unsigned done = 0;
  for (unsigned it = 0; it < kWaitLimit; ++it) {
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  atomicExch(err, 1);
  return false;
}

// LIST: the batch is the points pidx[0 .. min(npts, *pcount)) of the arrays (the gated
// surrogate's fallback list, whose length is known only on the device); otherwise points
// 0 .. npts. Either way each point's arithmetic is the same.
template <int BLOCK, int MINB, int AS, bool TMA, bool LIST = false>
__global__ void __launch_bounds__(BLOCK, MINB) snl1_band_kernel(
    const Snl1Dev p, int npts, const float* __restrict__ a, const float* __restrict__ cg,
    const float* __restrict__ kdmean, float* __restrict__ s, float* __restrict__ d,
    int* __restrict__ err, const int* __restrict__ pidx, const int* __restrict__ pcount) {
  extern __shared__ __align__(16) float smem[];
  if (LIST) npts = min(npts, __ldg(pcount));
  auto pt = [&](int i) { return LIST ? __ldg(pidx + i) : i; };
  const int nth = p.nth, nfr = p.nfr, nfrhgh = p.nfrhgh, nfrchg = p.nfrchg;
  const int nspec = p.nspec, nk = p.nk;
  // The six interaction arrays sit AS floats apart (AS >= (NFRCHG + 1) * NTH, a compile-time
  // stride), so one shared offset per (row, column) addresses all six with immediate offsets.
  float* const ue = smem;
  float* const arrs = ue + (nfrhgh + 1) * nth;
  float* const sa1 = arrs;
  float* const sa2 = arrs + AS;
  float* const da1p = arrs + 2 * AS;
  float* const da1m = arrs + 3 * AS;
  float* const da2p = arrs + 4 * AS;
  float* const da2m = arrs + 5 * AS;
  float* const dcs = arrs + 6 * AS;
  float* const conx2 = dcs + nspec;
  float* const afr = conx2 + 2 * nk;
  const size_t stage_off = (static_cast<size_t>(afr + nfrchg - smem) + 3) & ~static_cast<size_t>(3);
  float* const stage = smem + stage_off;
  uint64_t* const bar = reinterpret_cast<uint64_t*>(stage + ((nspec + nk + 3) & ~3));
  const int tid = threadIdx.x;

  // Once per CTA: zero rows, AF11 rows, the mbarrier and the first point's bulk copy.
  for (int i = tid; i < nth; i += BLOCK) {
    ue[i] = 0.0f;
    sa1[i] = sa2[i] = da1p[i] = da1m[i] = da2p[i] = da2m[i] = 0.0f;
  }
  for (int i = tid; i < nfrchg; i += BLOCK) afr[i] = p.af11_row[i];
  if (TMA && tid == 0) {
    mbar_init(bar, 1);
    if (blockIdx.x < npts) tma_fetch_point(bar, stage, a, cg, pt(blockIdx.x), nspec, nk);
  }
  __syncthreads();

  // This thread's column, band and wrapped columns.
  const int G = BLOCK / nth;
  const int ith = tid % nth, band = tid / nth;
  const bool active = band < G;
  const int br = (nfrchg + G - 1) / G;  // rows per band
  const int f0 = 1 + band * br;
  const int n3 = active ? max(0, min(br, nfrchg - f0 + 1)) : 0;
  const int n4 = active ? max(0, min(br, nfr - f0 + 1)) : 0;
  const int c0 = wrapc(ith + p.shift[0], nth), c1 = wrapc(ith + p.shift[1], nth);
  const int c2 = wrapc(ith + p.shift[2], nth), c3 = wrapc(ith + p.shift[3], nth);
  const int c4 = wrapc(ith + p.shift[4], nth), c5 = wrapc(ith + p.shift[5], nth);
  const int c6 = wrapc(ith + p.shift[6], nth), c7 = wrapc(ith + p.shift[7], nth);
  const int ifrp = p.ifrp, ifrm = p.ifrm;
  const float dal1 = p.dal1, dal2 = p.dal2, dal3 = p.dal3;
  // The UE loop of section 2 walks bins isp = tid + k * BLOCK.
  const int dq = BLOCK / nth, dr = BLOCK % nth, q0 = tid / nth, r0 = tid % nth;

  float kd_next = (blockIdx.x < npts) ? __ldg(kdmean + pt(blockIdx.x)) : 0.0f;
  unsigned parity = 0;
  int buf = 0;
  for (int ipt0 = blockIdx.x; ipt0 < npts; ipt0 += gridDim.x, buf ^= 1) {
    const int ipt = pt(ipt0);
    const float* const src_a = TMA ? stage : a + static_cast<size_t>(ipt) * nspec;
    const float* const src_c = TMA ? stage + nspec : cg + static_cast<size_t>(ipt) * nk;
    float* const conx = conx2 + buf * nk;
    bool lost = false;
    if (TMA) {
      lost = !mbar_wait(bar, parity, err);
      parity ^= 1u;
    }
    // 1. CONS; 2a. CON per frequency row.
    const float cons = dia_cons(p, kd_next);
    for (int k = tid; k < nk; k += BLOCK) conx[k] = kTpiInv / __ldg(p.sig + k) * src_c[k];
    // A bulk copy whose wait gave up ends this CTA's work here, all its threads together, so no
    // later copy is started on a barrier whose phase did not complete.
    if (__syncthreads_or(lost)) break;

    // 2b. UE = A / CON, and the parametric tail up each column from row NFR.
    {
      int ifr0 = q0, col = r0;
      for (int isp = tid; isp < nspec; isp += BLOCK) {
        const float v = (TMA ? src_a[isp] : __ldcs(src_a + isp)) / conx[ifr0];
        ue[isp + nth] = v;
        if (ifr0 == nfr - 1) {
          float t = v;
          for (int r = nfr + 1; r <= nfrhgh; ++r) {
            t = t * p.fachfe;
            ue[r * nth + col] = t;
          }
        }
        col += dr;
        ifr0 += dq;
        if (col >= nth) {
          col -= nth;
          ++ifr0;
        }
      }
    }
    __syncthreads();

    // The next point's A and CG stream into the staging buffer while this one is computed.
    const int inext = ipt0 + gridDim.x;
    if (TMA && tid == 0 && inext < npts) tma_fetch_point(bar, stage, a, cg, pt(inext), nspec, nk);
    if (inext < npts) kd_next = __ldg(kdmean + pt(inext));

    // 3. Interactions over the extended spectrum, sliding up the band.
    if (n3 > 0) {
      float pa[4], pb[4], ma[4], mb[4];  // plus rows: c1 c2 c5 c6; minus rows: c3 c4 c7 c8
#define WWB_LOAD_P(ROW, W)                    \
  {                                           \
    const int b_ = (ROW) * nth;               \
    W[0] = ue[b_ + c0];                       \
    W[1] = ue[b_ + c1];                       \
    W[2] = ue[b_ + c4];                       \
    W[3] = ue[b_ + c5];                       \
  }
#define WWB_LOAD_M(ROW, W)                    \
  {                                           \
    const int r_ = (ROW);                     \
    const int b_ = (r_ > 0 ? r_ : 0) * nth;   \
    W[0] = ue[b_ + c2];                       \
    W[1] = ue[b_ + c3];                       \
    W[2] = ue[b_ + c6];                       \
    W[3] = ue[b_ + c7];                       \
  }
      WWB_LOAD_P(f0 + ifrp, pa)
      WWB_LOAD_P(f0 + ifrp + 1, pb)
      WWB_LOAD_M(f0 + ifrm, ma)
      WWB_LOAD_M(f0 + ifrm - 1, mb)
#pragma unroll 1
      for (int k = 0; k < n3; ++k) {
        {
          const int f = f0 + k;
          const int o = f * nth + ith;
          const float e00 = ue[o];
          const float ep1 = p.awg[0] * pb[1] + p.awg[1] * pb[0] + p.awg[2] * pa[1] + p.awg[3] * pa[0];
          const float em1 = p.awg[4] * mb[3] + p.awg[5] * mb[2] + p.awg[6] * ma[3] + p.awg[7] * ma[2];
          const float ep2 = p.awg[0] * pb[3] + p.awg[1] * pb[2] + p.awg[2] * pa[3] + p.awg[3] * pa[2];
          const float em2 = p.awg[4] * mb[1] + p.awg[5] * mb[0] + p.awg[6] * ma[1] + p.awg[7] * ma[0];
          const float ca = cons * afr[f - 1];
          const float factor = ca * e00;
          const float sa1a = e00 * (ep1 * dal1 + em1 * dal2);
          const float sa1b = sa1a - ep1 * em1 * dal3;
          const float sa2a = e00 * (ep2 * dal1 + em2 * dal2);
          const float sa2b = sa2a - ep2 * em2 * dal3;
          const float v1 = factor * sa1b;
          const float v2 = factor * sa2b;
          sa1[o] = v1;
          sa2[o] = v2;
          if (f <= nfr) dcs[o - nth] = ca * (sa1a + sa1b) + ca * (sa2a + sa2b);
          da1p[o] = factor * (dal1 * e00 - dal3 * em1);
          da1m[o] = factor * (dal2 * e00 - dal3 * ep1);
          da2p[o] = factor * (dal1 * e00 - dal3 * em2);
          da2m[o] = factor * (dal2 * e00 - dal3 * ep2);
          if (k + 1 < n3) {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              pa[j] = pb[j];
              mb[j] = ma[j];
            }
            WWB_LOAD_P(f + 1 + ifrp + 1, pb)
            WWB_LOAD_M(f + 1 + ifrm, ma)
          }
        }
      }
    }
    __syncthreads();

    // 4. Source and diagonal terms, sliding up the band: S in one pass, D in a second, so each
    //    pass holds one set of windows (lo rows IF5/IF6: columns c5 c6 of SA1 or DA1P and c1 c2
    //    of SA2 or DA2P; hi rows IF7/IF8: c3 c4 of SA1 or DA1M and c7 c8 of SA2 or DA2M).
    if (n4 > 0) {
#define WWB_LO(A1, A2, ROW, W)                \
  {                                           \
    const int r_ = (ROW);                     \
    const int b_ = (r_ > 0 ? r_ : 0) * nth;   \
    W[0] = A1[b_ + c4];                       \
    W[1] = A1[b_ + c5];                       \
    W[2] = A2[b_ + c0];                       \
    W[3] = A2[b_ + c1];                       \
  }
#define WWB_HI(A1, A2, ROW, W)                \
  {                                           \
    const int b_ = (ROW) * nth;               \
    W[0] = A1[b_ + c2];                       \
    W[1] = A1[b_ + c3];                       \
    W[2] = A2[b_ + c6];                       \
    W[3] = A2[b_ + c7];                       \
  }
      float l5[4], l6[4], h7[4], h8[4];
      {
        float* const sp = s + static_cast<size_t>(ipt) * nspec;
        WWB_LO(sa1, sa2, f0 - ifrp, l5)
        WWB_LO(sa1, sa2, f0 - ifrp - 1, l6)
        WWB_HI(sa1, sa2, f0 - ifrm, h7)
        WWB_HI(sa1, sa2, f0 - ifrm + 1, h8)
#pragma unroll 1
        for (int k = 0; k < n4; ++k) {
          const int f = f0 + k;
          const int isp = (f - 1) * nth + ith;
          const float sv = conx[f - 1] * (-2.0f * (sa1[isp + nth] + sa2[isp + nth]) +
                                          p.awg[0] * (l6[1] + l6[3]) + p.awg[1] * (l6[0] + l6[2]) +
                                          p.awg[2] * (l5[1] + l5[3]) + p.awg[3] * (l5[0] + l5[2]) +
                                          p.awg[4] * (h8[1] + h8[3]) + p.awg[5] * (h8[0] + h8[2]) +
                                          p.awg[6] * (h7[1] + h7[3]) + p.awg[7] * (h7[0] + h7[2]));
          __stcs(sp + isp, sv);
          if (k + 1 < n4) {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              l6[j] = l5[j];
              h7[j] = h8[j];
            }
            WWB_LO(sa1, sa2, f + 1 - ifrp, l5)
            WWB_HI(sa1, sa2, f + 1 - ifrm + 1, h8)
          }
        }
      }
      {
        float* const dp = d + static_cast<size_t>(ipt) * nspec;
        WWB_LO(da1p, da2p, f0 - ifrp, l5)
        WWB_LO(da1p, da2p, f0 - ifrp - 1, l6)
        WWB_HI(da1m, da2m, f0 - ifrm, h7)
        WWB_HI(da1m, da2m, f0 - ifrm + 1, h8)
#pragma unroll 1
        for (int k = 0; k < n4; ++k) {
          const int f = f0 + k;
          const int isp = (f - 1) * nth + ith;
          const float dv = -2.0f * dcs[isp] +
                           p.swg[0] * (l6[1] + l6[3]) + p.swg[1] * (l6[0] + l6[2]) +
                           p.swg[2] * (l5[1] + l5[3]) + p.swg[3] * (l5[0] + l5[2]) +
                           p.swg[4] * (h8[1] + h8[3]) + p.swg[5] * (h8[0] + h8[2]) +
                           p.swg[6] * (h7[1] + h7[3]) + p.swg[7] * (h7[0] + h7[2]);
          __stcs(dp + isp, dv);
          if (k + 1 < n4) {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              l6[j] = l5[j];
              h7[j] = h8[j];
            }
            WWB_LO(da1p, da2p, f + 1 - ifrp, l5)
            WWB_HI(da1m, da2m, f + 1 - ifrm + 1, h8)
          }
        }
      }
#undef WWB_LO
#undef WWB_HI
    }
    // The next point's barriers order its writes of UE and the arrays after this section 4.
  }
#undef WWB_LOAD_P
#undef WWB_LOAD_M
}

// ------------------------------------------------------------------------------------------
// Tile kernel: the band kernel with the direction count NTH and the band height BR known at
// compile time, for the grids that dominate (36 directions, 8 bands of 5 rows; 24 directions,
// 12 bands of 3 rows).
//
// Every matrix gets PAD extra zero rows below row 0 (PAD >= MAX(IFRP, -IFRM)), so the clamped
// rows MAX(0, IFR + IFRM) etc. of INSNL1 read zeros without a clamp: the rows a band touches are
// then affine in its first row, each thread keeps one shared-memory pointer per (array group,
// wrapped column) and every access in the unrolled row loops is that pointer plus a
// compile-time offset. The arithmetic of each bin is the reference's, as in the other kernels.
template <int NTH, int G, int BR>
struct TileShape {
  static constexpr int kBlock = NTH * G;
  static constexpr int kPad = 4;                      // zero rows below row 0
  static constexpr int kRows = G * BR;                // rows the bands cover (>= NFRCHG)
  static constexpr int kAS = (kRows + 1 + kPad) * NTH;  // interaction-array stride
};

template <int NTH, int G, int BR, int MINB>
__global__ void __launch_bounds__(NTH * G, MINB) snl1_tile_kernel(
    const Snl1Dev p, const int npts, const float* __restrict__ a, const float* __restrict__ cg,
    const float* __restrict__ kdmean, float* __restrict__ s, float* __restrict__ d,
    int* __restrict__ err) {
  using S = TileShape<NTH, G, BR>;
  constexpr int BLOCK = S::kBlock, PAD = S::kPad, AS = S::kAS;
  extern __shared__ __align__(16) float smem[];
  const int nfr = p.nfr, nfrhgh = p.nfrhgh, nfrchg = p.nfrchg, nspec = p.nspec, nk = p.nk;
  const int ulen = (nfrhgh + 1 + PAD) * NTH;
  float* const ue = smem;  // row r at ue + (r + PAD) * NTH
  float* const arrs = ue + ((ulen + 3) & ~3);
  float* const sa1 = arrs;
  float* const sa2 = arrs + AS;
  float* const da1p = arrs + 2 * AS;
  float* const da1m = arrs + 3 * AS;
  float* const da2p = arrs + 4 * AS;
  float* const da2m = arrs + 5 * AS;
  float* const dcs = arrs + 6 * AS;        // rows 1..G*BR, row r at dcs + (r - 1) * NTH
  float* const conx2 = dcs + S::kRows * NTH;
  float* const afr = conx2 + ((2 * nk + 3) & ~3);
  float* const stage = afr + ((nfrchg + 3) & ~3);  // 16-byte aligned: every offset above is
  uint64_t* const bar = reinterpret_cast<uint64_t*>(stage + ((nspec + nk + 3) & ~3));
  const int tid = threadIdx.x;

  // Once per CTA: the zero rows (PAD below row 0, and row 0) of UE and the six arrays.
  for (int i = tid; i < (PAD + 1) * NTH; i += BLOCK) {
    ue[i] = 0.0f;
#pragma unroll
    for (int j = 0; j < 6; ++j) arrs[j * AS + i] = 0.0f;
  }
  for (int i = tid; i < nfrchg; i += BLOCK) afr[i] = p.af11_row[i];
  if (tid == 0) {
    mbar_init(bar, 1);
    if (blockIdx.x < npts) tma_fetch_point(bar, stage, a, cg, blockIdx.x, nspec, nk);
  }
  __syncthreads();

  const int ith = tid % NTH, band = tid / NTH;
  const int f0 = 1 + band * BR;
  const int n3 = max(0, min(BR, nfrchg - f0 + 1));
  const int n4 = max(0, min(BR, nfr - f0 + 1));
  const int c0 = wrapc(ith + p.shift[0], NTH), c1 = wrapc(ith + p.shift[1], NTH);
  const int c2 = wrapc(ith + p.shift[2], NTH), c3 = wrapc(ith + p.shift[3], NTH);
  const int c4 = wrapc(ith + p.shift[4], NTH), c5 = wrapc(ith + p.shift[5], NTH);
  const int c6 = wrapc(ith + p.shift[6], NTH), c7 = wrapc(ith + p.shift[7], NTH);
  const int ifrp = p.ifrp, ifrm = p.ifrm;
  const float dal1 = p.dal1, dal2 = p.dal2, dal3 = p.dal3;
  // Row bases (in floats, PAD included) of this thread's band.
  const int rP = (f0 + ifrp + PAD) * NTH;      // IF1 of the band's first row
  const int rM = (f0 + ifrm - 1 + PAD) * NTH;  // IF4 of the band's first row
  const int rO = (f0 + PAD) * NTH + ith;       // the band's own bins
  const int rL = (f0 - ifrp - 1 + PAD) * NTH;  // IF6 of the band's first row
  const int rH = (f0 - ifrm + PAD) * NTH;      // IF7 of the band's first row

  float kd_next = (blockIdx.x < npts) ? __ldg(kdmean + blockIdx.x) : 0.0f;
  unsigned parity = 0;
  int buf = 0;
  for (int ipt = blockIdx.x; ipt < npts; ipt += gridDim.x, buf ^= 1) {
    float* const conx = conx2 + buf * nk;
    const bool lost = !mbar_wait(bar, parity, err);
    parity ^= 1u;
    const float cons = dia_cons(p, kd_next);
    for (int k = tid; k < nk; k += BLOCK) conx[k] = kTpiInv / __ldg(p.sig + k) * stage[nspec + k];
    if (__syncthreads_or(lost)) break;  // as in the band kernel: stop together, fetch no more
    // 2b. UE = A / CON, and the parametric tail up each column from row NFR.
    for (int isp = tid; isp < nspec; isp += BLOCK) {
      const int ifr0 = isp / NTH, col = isp - ifr0 * NTH;
      const float v = stage[isp] / conx[ifr0];
      ue[(ifr0 + 1 + PAD) * NTH + col] = v;
      if (ifr0 == nfr - 1) {
        float t = v;
        for (int r = nfr + 1; r <= nfrhgh; ++r) {
          t = t * p.fachfe;
          ue[(r + PAD) * NTH + col] = t;
        }
      }
    }
    __syncthreads();
    const int inext = ipt + gridDim.x;
    if (tid == 0 && inext < npts) tma_fetch_point(bar, stage, a, cg, inext, nspec, nk);
    if (inext < npts) kd_next = __ldg(kdmean + inext);

    // 3. Interactions, rows f0 .. f0+BR-1 of the band.
    {
      float pw[BR + 2][4];  // IF1/IF2 rows: columns c0 c1 c4 c5
      float mw[BR + 1][4];  // IF4/IF3 rows: columns c2 c3 c6 c7
      // Rows enter the windows one step ahead of their use, so at most three of each are live.
#define WWB_LOAD_PW(j)                          \
  {                                             \
    const float* u = ue + rP + (j) * NTH;       \
    pw[j][0] = u[c0];                           \
    pw[j][1] = u[c1];                           \
    pw[j][2] = u[c4];                           \
    pw[j][3] = u[c5];                           \
  }
#define WWB_LOAD_MW(j)                          \
  {                                             \
    const float* u = ue + rM + (j) * NTH;       \
    mw[j][0] = u[c2];                           \
    mw[j][1] = u[c3];                           \
    mw[j][2] = u[c6];                           \
    mw[j][3] = u[c7];                           \
  }
      if (n3 > 0) {
        WWB_LOAD_PW(0);
        WWB_LOAD_MW(0);
      }
#pragma unroll
      for (int k = 0; k < BR; ++k) {
        if (k < n3) {
          WWB_LOAD_PW(k + 1);
          WWB_LOAD_MW(k + 1);
#define pa pw[k]       // IF1 row
#define pb pw[k + 1]   // IF2 row
#define mb mw[k]       // IF4 row
#define ma mw[k + 1]   // IF3 row
          const int o = rO + k * NTH;
          const float e00 = ue[o];
          const float ep1 = p.awg[0] * pb[1] + p.awg[1] * pb[0] + p.awg[2] * pa[1] + p.awg[3] * pa[0];
          const float em1 = p.awg[4] * mb[3] + p.awg[5] * mb[2] + p.awg[6] * ma[3] + p.awg[7] * ma[2];
          const float ep2 = p.awg[0] * pb[3] + p.awg[1] * pb[2] + p.awg[2] * pa[3] + p.awg[3] * pa[2];
          const float em2 = p.awg[4] * mb[1] + p.awg[5] * mb[0] + p.awg[6] * ma[1] + p.awg[7] * ma[0];
          const float ca = cons * afr[f0 - 1 + k];
          const float factor = ca * e00;
          const float sa1a = e00 * (ep1 * dal1 + em1 * dal2);
          const float sa1b = sa1a - ep1 * em1 * dal3;
          const float sa2a = e00 * (ep2 * dal1 + em2 * dal2);
          const float sa2b = sa2a - ep2 * em2 * dal3;
          sa1[o] = factor * sa1b;
          sa2[o] = factor * sa2b;
          if (f0 + k <= nfr) dcs[o - (PAD + 1) * NTH] = ca * (sa1a + sa1b) + ca * (sa2a + sa2b);
          da1p[o] = factor * (dal1 * e00 - dal3 * em1);
          da1m[o] = factor * (dal2 * e00 - dal3 * ep1);
          da2p[o] = factor * (dal1 * e00 - dal3 * em2);
          da2m[o] = factor * (dal2 * e00 - dal3 * ep2);
#undef pa
#undef pb
#undef mb
#undef ma
        }
      }
#undef WWB_LOAD_PW
#undef WWB_LOAD_MW
    }
    __syncthreads();

    // 4. Source and diagonal terms, rows f0 .. f0+BR-1 of the band (up to NFR).
    {
      float* const sp = s + static_cast<size_t>(ipt) * nspec + (f0 - 1) * NTH + ith;
      float* const dp = d + static_cast<size_t>(ipt) * nspec + (f0 - 1) * NTH + ith;
      float lw[BR + 1][4], hw[BR + 1][4];  // lo rows IF6.. (SA1 c4 c5, SA2 c0 c1); hi rows IF7..
#define WWB_LOAD_LH(j, L1, L2, H1, H2)           \
  {                                              \
    const int bl = rL + (j) * NTH, bh = rH + (j) * NTH; \
    lw[j][0] = L1[bl + c4];                      \
    lw[j][1] = L1[bl + c5];                      \
    lw[j][2] = L2[bl + c0];                      \
    lw[j][3] = L2[bl + c1];                      \
    hw[j][0] = H1[bh + c2];                      \
    hw[j][1] = H1[bh + c3];                      \
    hw[j][2] = H2[bh + c6];                      \
    hw[j][3] = H2[bh + c7];                      \
  }
      if (n4 > 0) WWB_LOAD_LH(0, sa1, sa2, sa1, sa2);
#pragma unroll
      for (int k = 0; k < BR; ++k) {
        if (k < n4) {
          WWB_LOAD_LH(k + 1, sa1, sa2, sa1, sa2);
#define l6 lw[k]
#define l5 lw[k + 1]
#define h7 hw[k]
#define h8 hw[k + 1]
          const int o = rO + k * NTH;
          const float sv = conx[f0 - 1 + k] * (-2.0f * (sa1[o] + sa2[o]) +
                                               p.awg[0] * (l6[1] + l6[3]) + p.awg[1] * (l6[0] + l6[2]) +
                                               p.awg[2] * (l5[1] + l5[3]) + p.awg[3] * (l5[0] + l5[2]) +
                                               p.awg[4] * (h8[1] + h8[3]) + p.awg[5] * (h8[0] + h8[2]) +
                                               p.awg[6] * (h7[1] + h7[3]) + p.awg[7] * (h7[0] + h7[2]));
          __stcs(sp + k * NTH, sv);
#undef l6
#undef l5
#undef h7
#undef h8
        }
      }
      if (n4 > 0) WWB_LOAD_LH(0, da1p, da2p, da1m, da2m);
#pragma unroll
      for (int k = 0; k < BR; ++k) {
        if (k < n4) {
          WWB_LOAD_LH(k + 1, da1p, da2p, da1m, da2m);
#define l6 lw[k]
#define l5 lw[k + 1]
#define h7 hw[k]
#define h8 hw[k + 1]
          const float dv = -2.0f * dcs[rO - (PAD + 1) * NTH + k * NTH] +
                           p.swg[0] * (l6[1] + l6[3]) + p.swg[1] * (l6[0] + l6[2]) +
                           p.swg[2] * (l5[1] + l5[3]) + p.swg[3] * (l5[0] + l5[2]) +
                           p.swg[4] * (h8[1] + h8[3]) + p.swg[5] * (h8[0] + h8[2]) +
                           p.swg[6] * (h7[1] + h7[3]) + p.swg[7] * (h7[0] + h7[2]);
          __stcs(dp + k * NTH, dv);
#undef l6
#undef l5
#undef h7
#undef h8
        }
      }
#undef WWB_LOAD_LH
    }
    // The next point's two barriers order its writes after this section 4.
  }
}

// ------------------------------------------------------------------------------------------
// Pair kernel: the band kernel over two sea points at once.
//
// The two points of a pair share every index: the same bins, rows, wrapped columns and table
// entries. So each shared-memory slot holds both points' values side by side (a float2: .x the
// first point, .y the second), each window load is one 64-bit load for both, and the additions
// of the reference are paired FADD2 (__fadd2_rn: per component the IEEE addition of
// __fadd_rn). Every component follows its own point's expression in the reference's order
// (snl1_team.hpp:383-496), so the results are those of the band kernel bit for bit while the
// instructions issued per point drop. A - B is A + (-B), the same IEEE result.
//
// One rule keeps the pairs exact: a product that feeds an addition is formed by two scalar
// __fmul_rn (mulS), never by a paired multiply. Measured on B200 with this toolchain, a paired
// multiply (__fmul2_rn, or mul.rn.f32x2 / fma.rn.f32x2 with a -0 addend in inline PTX) whose
// result feeds a paired addition came out as a fused multiply-add in 21 % of 2^20 random cases
// (and in 39 % of the S values of 1000 sea states), whatever -fmad says, while each paired
// operation alone, and scalar products summed by paired additions, matched the scalar IEEE
// operations on every case. Paired multiplies (mul2) are used only where the product feeds
// another multiply or is stored.
//
// Shared memory (float2 unless noted): UE rows 0..NFRHGH; SA1, SA2, DA1P, DA1M, DA2P, DA2M (AS
// float2 apart); DC over NSPEC bins; CON rows (2 x NK, double-buffered by pair parity); CONS of
// the two points (2, by parity); AF11 rows (NFRCHG floats); the staging buffer (A of both points,
// then CG of both, floats); the mbarrier. An odd last point is paired with itself and stored once.
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
  return __fadd2_rn(a, make_float2(-b.x, -b.y));
}
__device__ __forceinline__ float2 dup2(float v) { return make_float2(v, v); }
/// A product that feeds an addition: two scalar IEEE multiplies (see above).
__device__ __forceinline__ float2 mulS(float2 a, float2 b) {
  return make_float2(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y));
}

/// One elected thread: expect the bytes of two points and start the four bulk copies.
__device__ __forceinline__ void tma_fetch_pair(uint64_t* bar, float* stage, const float* a,
                                               const float* cg, int i0, int i1, int nspec,
                                               int nk, unsigned extra = 0) {
  const unsigned bytes_a = static_cast<unsigned>(nspec) * 4u;
  const unsigned bytes_c = static_cast<unsigned>(nk) * 4u;
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(2u * (bytes_a + bytes_c) + extra)
               : "memory");
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const int ip = j == 0 ? i0 : i1;
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_u32(stage + j * nspec)),
        "l"(a + static_cast<size_t>(ip) * nspec), "r"(bytes_a), "r"(smem_u32(bar))
        : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_u32(stage + 2 * nspec + j * nk)),
        "l"(cg + static_cast<size_t>(ip) * nk), "r"(bytes_c), "r"(smem_u32(bar))
        : "memory");
  }
}

template <int BLOCK, int MINB, int AS, bool LIST>
__global__ void __launch_bounds__(BLOCK, MINB) snl1_pair_kernel(
    const Snl1Dev p, int npts, const float* __restrict__ a, const float* __restrict__ cg,
    const float* __restrict__ kdmean, float* __restrict__ s, float* __restrict__ d,
    int* __restrict__ err, const int* __restrict__ pidx, const int* __restrict__ pcount) {
  extern __shared__ __align__(16) float smem[];
  if (LIST) npts = min(npts, __ldg(pcount));
  auto pt = [&](int i) { return LIST ? __ldg(pidx + i) : i; };
  const int npairs = (npts + 1) >> 1;
  const int nth = p.nth, nfr = p.nfr, nfrhgh = p.nfrhgh, nfrchg = p.nfrchg;
  const int nspec = p.nspec, nk = p.nk;
  float2* const ue = reinterpret_cast<float2*>(smem);
  float2* const arrs = ue + (nfrhgh + 1) * nth;
  float2* const sa1 = arrs;
  float2* const sa2 = arrs + AS;
  float2* const da1p = arrs + 2 * AS;
  float2* const da1m = arrs + 3 * AS;
  float2* const da2p = arrs + 4 * AS;
  float2* const da2m = arrs + 5 * AS;
  float2* const dcs = arrs + 6 * AS;
  float2* const conx2 = dcs + nspec;
  float2* const cons2 = conx2 + 2 * nk;
  float* const afr = reinterpret_cast<float*>(cons2 + 2);
  const size_t stage_off =
      (static_cast<size_t>(afr + nfrchg - smem) + 3) & ~static_cast<size_t>(3);
  float* const stage = smem + stage_off;
  uint64_t* const bar = reinterpret_cast<uint64_t*>(stage + ((2 * (nspec + nk) + 3) & ~3));
  const int tid = threadIdx.x;

  // The points of pair pp: 2 pp and 2 pp + 1 of the batch (an odd last point twice).
  auto first_of = [&](int pp) { return pt(2 * pp); };
  auto second_of = [&](int pp) { return 2 * pp + 1 < npts ? pt(2 * pp + 1) : pt(2 * pp); };

  for (int i = tid; i < nth; i += BLOCK) {
    const float2 z = make_float2(0.0f, 0.0f);
    ue[i] = z;
    sa1[i] = sa2[i] = da1p[i] = da1m[i] = da2p[i] = da2m[i] = z;
  }
  for (int i = tid; i < nfrchg; i += BLOCK) afr[i] = p.af11_row[i];
  float kd0 = 0.0f, kd1 = 0.0f;  // thread 0: the KDMEAN of its CTA's next pair
  if (tid == 0) {
    mbar_init(bar, 1);
    if (blockIdx.x < npairs) {
      const int i0 = first_of(blockIdx.x), i1 = second_of(blockIdx.x);
      tma_fetch_pair(bar, stage, a, cg, i0, i1, nspec, nk, static_cast<unsigned>(p.stall_tx));
      kd0 = __ldg(kdmean + i0);
      kd1 = __ldg(kdmean + i1);
    }
  }
  __syncthreads();

  const int G = BLOCK / nth;
  const int ith = tid % nth, band = tid / nth;
  const bool active = band < G;
  const int br = (nfrchg + G - 1) / G;
  const int f0 = 1 + band * br;
  const int n3 = active ? max(0, min(br, nfrchg - f0 + 1)) : 0;
  const int n4 = active ? max(0, min(br, nfr - f0 + 1)) : 0;
  const int c0 = wrapc(ith + p.shift[0], nth), c1 = wrapc(ith + p.shift[1], nth);
  const int c2 = wrapc(ith + p.shift[2], nth), c3 = wrapc(ith + p.shift[3], nth);
  const int c4 = wrapc(ith + p.shift[4], nth), c5 = wrapc(ith + p.shift[5], nth);
  const int c6 = wrapc(ith + p.shift[6], nth), c7 = wrapc(ith + p.shift[7], nth);
  const int ifrp = p.ifrp, ifrm = p.ifrm;
  const int dq = BLOCK / nth, dr = BLOCK % nth, q0 = tid / nth, r0 = tid % nth;

  unsigned parity = 0;
  int buf = 0;
  for (int pp = blockIdx.x; pp < npairs; pp += gridDim.x, buf ^= 1) {
    const int i0 = first_of(pp), i1 = second_of(pp);
    const bool has1 = 2 * pp + 1 < npts;
    float2* const conx = conx2 + buf * nk;
    const bool lost = !mbar_wait(bar, parity, err);
    parity ^= 1u;
    // 1. CONS of both points (one thread); 2a. CON per frequency row.
    if (tid == 0) cons2[buf] = make_float2(dia_cons(p, kd0), dia_cons(p, kd1));
    for (int k = tid; k < nk; k += BLOCK) {
      const float w = kTpiInv / __ldg(p.sig + k);
      conx[k] = make_float2(w * stage[2 * nspec + k], w * stage[2 * nspec + nk + k]);
    }
    // A bulk copy whose wait gave up ends this CTA's work here, all its threads together.
    if (__syncthreads_or(lost)) break;

    // 2b. UE = A / CON, and the parametric tail up each column from row NFR.
    {
      int ifr0 = q0, col = r0;
      for (int isp = tid; isp < nspec; isp += BLOCK) {
        const float2 cx = conx[ifr0];
        const float2 v = make_float2(stage[isp] / cx.x, stage[nspec + isp] / cx.y);
        ue[isp + nth] = v;
        if (ifr0 == nfr - 1) {
          float2 t = v;
          const float2 fh = dup2(p.fachfe);
          for (int r = nfr + 1; r <= nfrhgh; ++r) {
            t = mul2(t, fh);
            ue[r * nth + col] = t;
          }
        }
        col += dr;
        ifr0 += dq;
        if (col >= nth) {
          col -= nth;
          ++ifr0;
        }
      }
    }
    __syncthreads();

    // The next pair's A and CG stream into the staging buffer while this one is computed.
    const int pnext = pp + gridDim.x;
    if (tid == 0 && pnext < npairs) {
      const int j0 = first_of(pnext), j1 = second_of(pnext);
      tma_fetch_pair(bar, stage, a, cg, j0, j1, nspec, nk);
      kd0 = __ldg(kdmean + j0);
      kd1 = __ldg(kdmean + j1);
    }
    const float2 cons = cons2[buf];

    // 3. Interactions over the extended spectrum, sliding up the band.
    if (n3 > 0) {
      const float2 w0 = dup2(p.awg[0]), w1 = dup2(p.awg[1]), w2 = dup2(p.awg[2]),
                   w3 = dup2(p.awg[3]), w4 = dup2(p.awg[4]), w5 = dup2(p.awg[5]),
                   w6 = dup2(p.awg[6]), w7 = dup2(p.awg[7]);
      const float2 dl1 = dup2(p.dal1), dl2 = dup2(p.dal2), dl3 = dup2(p.dal3);
      float2 pa[4], pb[4], ma[4], mb[4];  // plus rows: c1 c2 c5 c6; minus rows: c3 c4 c7 c8
#define WWB_P2(ROW, W)                        \
  {                                           \
    const int b_ = (ROW) * nth;               \
    W[0] = ue[b_ + c0];                       \
    W[1] = ue[b_ + c1];                       \
    W[2] = ue[b_ + c4];                       \
    W[3] = ue[b_ + c5];                       \
  }
#define WWB_M2(ROW, W)                        \
  {                                           \
    const int r_ = (ROW);                     \
    const int b_ = (r_ > 0 ? r_ : 0) * nth;   \
    W[0] = ue[b_ + c2];                       \
    W[1] = ue[b_ + c3];                       \
    W[2] = ue[b_ + c6];                       \
    W[3] = ue[b_ + c7];                       \
  }
      WWB_P2(f0 + ifrp, pa)
      WWB_P2(f0 + ifrp + 1, pb)
      WWB_M2(f0 + ifrm, ma)
      WWB_M2(f0 + ifrm - 1, mb)
#pragma unroll 1
      for (int k = 0; k < n3; ++k) {
        const int f = f0 + k;
        const int o = f * nth + ith;
        const float2 e00 = ue[o];
        const float2 ep1 = add2(add2(add2(mulS(w0, pb[1]), mulS(w1, pb[0])), mulS(w2, pa[1])),
                                mulS(w3, pa[0]));
        const float2 em1 = add2(add2(add2(mulS(w4, mb[3]), mulS(w5, mb[2])), mulS(w6, ma[3])),
                                mulS(w7, ma[2]));
        const float2 ep2 = add2(add2(add2(mulS(w0, pb[3]), mulS(w1, pb[2])), mulS(w2, pa[3])),
                                mulS(w3, pa[2]));
        const float2 em2 = add2(add2(add2(mulS(w4, mb[1]), mulS(w5, mb[0])), mulS(w6, ma[1])),
                                mulS(w7, ma[0]));
        const float2 ca = mul2(cons, dup2(afr[f - 1]));
        const float2 factor = mul2(ca, e00);
        const float2 sa1a = mulS(e00, add2(mulS(ep1, dl1), mulS(em1, dl2)));
        const float2 sa1b = sub2(sa1a, mulS(mul2(ep1, em1), dl3));
        const float2 sa2a = mulS(e00, add2(mulS(ep2, dl1), mulS(em2, dl2)));
        const float2 sa2b = sub2(sa2a, mulS(mul2(ep2, em2), dl3));
        sa1[o] = mul2(factor, sa1b);
        sa2[o] = mul2(factor, sa2b);
        if (f <= nfr) dcs[o - nth] = add2(mulS(ca, add2(sa1a, sa1b)), mulS(ca, add2(sa2a, sa2b)));
        da1p[o] = mul2(factor, sub2(mulS(dl1, e00), mulS(dl3, em1)));
        da1m[o] = mul2(factor, sub2(mulS(dl2, e00), mulS(dl3, ep1)));
        da2p[o] = mul2(factor, sub2(mulS(dl1, e00), mulS(dl3, em2)));
        da2m[o] = mul2(factor, sub2(mulS(dl2, e00), mulS(dl3, ep2)));
        if (k + 1 < n3) {
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            pa[j] = pb[j];
            mb[j] = ma[j];
          }
          WWB_P2(f + 1 + ifrp + 1, pb)
          WWB_M2(f + 1 + ifrm, ma)
        }
      }
#undef WWB_P2
#undef WWB_M2
    }
    __syncthreads();

    // 4. Source and diagonal terms (as the band kernel: S in one pass, D in a second).
    if (n4 > 0) {
#define WWB_LO2(A1, A2, ROW, W)               \
  {                                           \
    const int r_ = (ROW);                     \
    const int b_ = (r_ > 0 ? r_ : 0) * nth;   \
    W[0] = A1[b_ + c4];                       \
    W[1] = A1[b_ + c5];                       \
    W[2] = A2[b_ + c0];                       \
    W[3] = A2[b_ + c1];                       \
  }
#define WWB_HI2(A1, A2, ROW, W)               \
  {                                           \
    const int b_ = (ROW) * nth;               \
    W[0] = A1[b_ + c2];                       \
    W[1] = A1[b_ + c3];                       \
    W[2] = A2[b_ + c6];                       \
    W[3] = A2[b_ + c7];                       \
  }
      const float2 m2 = dup2(-2.0f);
      float2 l5[4], l6[4], h7[4], h8[4];
      {
        const float2 w0 = dup2(p.awg[0]), w1 = dup2(p.awg[1]), w2 = dup2(p.awg[2]),
                     w3 = dup2(p.awg[3]), w4 = dup2(p.awg[4]), w5 = dup2(p.awg[5]),
                     w6 = dup2(p.awg[6]), w7 = dup2(p.awg[7]);
        float* const sp0 = s + static_cast<size_t>(i0) * nspec;
        float* const sp1 = s + static_cast<size_t>(i1) * nspec;
        WWB_LO2(sa1, sa2, f0 - ifrp, l5)
        WWB_LO2(sa1, sa2, f0 - ifrp - 1, l6)
        WWB_HI2(sa1, sa2, f0 - ifrm, h7)
        WWB_HI2(sa1, sa2, f0 - ifrm + 1, h8)
#pragma unroll 1
        for (int k = 0; k < n4; ++k) {
          const int f = f0 + k;
          const int isp = (f - 1) * nth + ith;
          float2 t = mulS(m2, add2(sa1[isp + nth], sa2[isp + nth]));
          t = add2(t, mulS(w0, add2(l6[1], l6[3])));
          t = add2(t, mulS(w1, add2(l6[0], l6[2])));
          t = add2(t, mulS(w2, add2(l5[1], l5[3])));
          t = add2(t, mulS(w3, add2(l5[0], l5[2])));
          t = add2(t, mulS(w4, add2(h8[1], h8[3])));
          t = add2(t, mulS(w5, add2(h8[0], h8[2])));
          t = add2(t, mulS(w6, add2(h7[1], h7[3])));
          t = add2(t, mulS(w7, add2(h7[0], h7[2])));
          const float2 sv = mul2(conx[f - 1], t);
          __stcs(sp0 + isp, sv.x);
          if (has1) __stcs(sp1 + isp, sv.y);
          if (k + 1 < n4) {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              l6[j] = l5[j];
              h7[j] = h8[j];
            }
            WWB_LO2(sa1, sa2, f + 1 - ifrp, l5)
            WWB_HI2(sa1, sa2, f + 1 - ifrm + 1, h8)
          }
        }
      }
      {
        const float2 w0 = dup2(p.swg[0]), w1 = dup2(p.swg[1]), w2 = dup2(p.swg[2]),
                     w3 = dup2(p.swg[3]), w4 = dup2(p.swg[4]), w5 = dup2(p.swg[5]),
                     w6 = dup2(p.swg[6]), w7 = dup2(p.swg[7]);
        float* const dp0 = d + static_cast<size_t>(i0) * nspec;
        float* const dp1 = d + static_cast<size_t>(i1) * nspec;
        WWB_LO2(da1p, da2p, f0 - ifrp, l5)
        WWB_LO2(da1p, da2p, f0 - ifrp - 1, l6)
        WWB_HI2(da1m, da2m, f0 - ifrm, h7)
        WWB_HI2(da1m, da2m, f0 - ifrm + 1, h8)
#pragma unroll 1
        for (int k = 0; k < n4; ++k) {
          const int f = f0 + k;
          const int isp = (f - 1) * nth + ith;
          float2 t = mulS(m2, dcs[isp]);
          t = add2(t, mulS(w0, add2(l6[1], l6[3])));
          t = add2(t, mulS(w1, add2(l6[0], l6[2])));
          t = add2(t, mulS(w2, add2(l5[1], l5[3])));
          t = add2(t, mulS(w3, add2(l5[0], l5[2])));
          t = add2(t, mulS(w4, add2(h8[1], h8[3])));
          t = add2(t, mulS(w5, add2(h8[0], h8[2])));
          t = add2(t, mulS(w6, add2(h7[1], h7[3])));
          t = add2(t, mulS(w7, add2(h7[0], h7[2])));
          __stcs(dp0 + isp, t.x);
          if (has1) __stcs(dp1 + isp, t.y);
          if (k + 1 < n4) {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              l6[j] = l5[j];
              h7[j] = h8[j];
            }
            WWB_LO2(da1p, da2p, f + 1 - ifrp, l5)
            WWB_HI2(da1m, da2m, f + 1 - ifrm + 1, h8)
          }
        }
      }
#undef WWB_LO2
#undef WWB_HI2
    }
    // The next pair's barriers order its writes of UE and the arrays after this section 4.
  }
}

// ------------------------------------------------------------------------------------------
// Pair-tile kernel: the pair kernel with the direction count NTH, the band count G and the band
// height BR known at compile time (36 directions: 8 bands of 5 rows), every row loop unrolled.
// Each matrix has zero rows below row 0 (PADU for UE, PADA for the interaction arrays), so the
// clamped rows MAX(0, IFR + IFRM - 1) and MAX(0, IFR - IFRP - 1) of INSNL1 read zeros without a
// clamp (row 0 is zero too). Every row a thread touches is then its band's first row plus a
// compile-time offset: each window column keeps one shared-memory pointer, set once per thread,
// and every load and store in the unrolled rows is that pointer plus an immediate. Every band
// runs all BR rows in both sections with no branch (the tables fill G x BR rows of section 3
// exactly); section 4's rows above NFR are computed and not stored, their reads landing in the
// next matrix or in DC's slack rows. The arithmetic of each bin is the pair kernel's (and so the
// reference's), with the same rule for paired operations.
__device__ __forceinline__ float2 mulS1(float w, float2 x) {
  return make_float2(__fmul_rn(w, x.x), __fmul_rn(w, x.y));
}

template <int NTH, int G, int BR, int PADU, int PADA>
struct PairTileShape {
  static constexpr int kBlock = NTH * G;
  static constexpr int kRowsA = PADA + 1 + G * BR;  ///< interaction-array rows -PADA .. G BR
  static constexpr int kAS = kRowsA * NTH;          ///< float2 slots per interaction array
  static constexpr int kRowsU = PADU + 1 + G * BR + PADA + 1;  ///< UE rows -PADU .. G BR + PADA + 1
  static constexpr int kDcs = G * BR * NTH;  ///< DC slots: NSPEC and the rows above NFR
};

template <int NTH, int G, int BR, int PADU, int PADA, bool LIST>
__global__ void __launch_bounds__(NTH * G, 2) snl1_pairtile_kernel(
    const Snl1Dev p, int npts, const float* __restrict__ a, const float* __restrict__ cg,
    const float* __restrict__ kdmean, float* __restrict__ s, float* __restrict__ d,
    int* __restrict__ err, const int* __restrict__ pidx, const int* __restrict__ pcount) {
  using S = PairTileShape<NTH, G, BR, PADU, PADA>;
  constexpr int BLOCK = S::kBlock, AS = S::kAS;
  extern __shared__ __align__(16) float smem[];
  if (LIST) npts = min(npts, __ldg(pcount));
  auto pt = [&](int i) { return LIST ? __ldg(pidx + i) : i; };
  const int npairs = (npts + 1) >> 1;
  const int nfr = p.nfr, nfrchg = p.nfrchg, nspec = p.nspec, nk = p.nk;
  float2* const ue0 = reinterpret_cast<float2*>(smem);  // row -PADU
  float2* const ue = ue0 + PADU * NTH;                  // row 0
  float2* const arr0 = ue0 + S::kRowsU * NTH;           // SA1 row -PADA; the others AS apart
  float2* const arr = arr0 + PADA * NTH;                // SA1 row 0
  float2* const dcs = arr0 + 6 * AS;
  float2* const conx2 = dcs + S::kDcs;
  float2* const cons2 = conx2 + 2 * nk;
  float* const afr = reinterpret_cast<float*>(cons2 + 2);
  float* const wrow = afr + nfrchg;  // TPIINV / SIG per frequency row
  const size_t stage_off =
      (static_cast<size_t>(wrow + nk - smem) + 3) & ~static_cast<size_t>(3);
  float* const stage = smem + stage_off;
  uint64_t* const bar = reinterpret_cast<uint64_t*>(stage + ((2 * (nspec + nk) + 3) & ~3));
  const int tid = threadIdx.x;

  auto first_of = [&](int pp) { return pt(2 * pp); };
  auto second_of = [&](int pp) { return 2 * pp + 1 < npts ? pt(2 * pp + 1) : pt(2 * pp); };

  // Zero rows -PADU..0 of UE and -PADA..0 of the six arrays, once per CTA.
  {
    const float2 z = make_float2(0.0f, 0.0f);
    for (int i = tid; i < (PADU + 1) * NTH; i += BLOCK) ue0[i] = z;
    for (int i = tid; i < (PADA + 1) * NTH; i += BLOCK)
#pragma unroll
      for (int m = 0; m < 6; ++m) arr0[m * AS + i] = z;
  }
  for (int i = tid; i < nfrchg; i += BLOCK) afr[i] = p.af11_row[i];
  for (int i = tid; i < nk; i += BLOCK) wrow[i] = kTpiInv / __ldg(p.sig + i);
  if (tid == 0) {
    mbar_init(bar, 1);
    if (blockIdx.x < npairs) {
      const int i0 = first_of(blockIdx.x), i1 = second_of(blockIdx.x);
      tma_fetch_pair(bar, stage, a, cg, i0, i1, nspec, nk, static_cast<unsigned>(p.stall_tx));
    }
  }
  __syncthreads();

  const int ith = tid % NTH, band = tid / NTH;
  const int f0 = 1 + band * BR;
  const int ifrp = p.ifrp, ifrm = p.ifrm;
  int c[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) c[j] = wrapc(ith + p.shift[j], NTH);
  // Section 3: the bin's own row, the plus rows (IF1 = f + IFRP, IF2 = IF1 + 1; columns c0 c1
  // c4 c5) and the minus rows (IF4 = f + IFRM - 1, IF3 = IF4 + 1; columns c2 c3 c6 c7).
  const float2* const pe = ue + f0 * NTH + ith;
  const float2* const pp0 = ue + (f0 + ifrp) * NTH;
  const float2* const pm0 = ue + (f0 + ifrm - 1) * NTH;
  float2* const po = arr + f0 * NTH + ith;
  float2* const pd = dcs + (f0 - 1) * NTH + ith;
  // Section 4: the lo rows (IF6 = f - IFRP - 1, IF5 = IF6 + 1; columns c4 c5 of SA1/DA1P, c0 c1
  // of SA2/DA2P) and the hi rows (IF7 = f - IFRM, IF8 = IF7 + 1; columns c2 c3 of SA1/DA1M, c6 c7
  // of SA2/DA2M).
  const float2* const pl0 = arr + (f0 - ifrp - 1) * NTH;
  const float2* const ph0 = arr + (f0 - ifrm) * NTH;
  const float w0 = p.awg[0], w1 = p.awg[1], w2 = p.awg[2], w3 = p.awg[3];
  const float w4 = p.awg[4], w5 = p.awg[5], w6 = p.awg[6], w7 = p.awg[7];
  const float dal1 = p.dal1, dal2 = p.dal2, dal3 = p.dal3;
  constexpr int dq = BLOCK / NTH, dr = BLOCK % NTH;
  const int q0 = tid / NTH, r0 = tid % NTH;

  unsigned parity = 0;
  int buf = 0;
  for (int pp = blockIdx.x; pp < npairs; pp += gridDim.x, buf ^= 1) {
    const int i0 = first_of(pp), i1 = second_of(pp);
    const bool has1 = 2 * pp + 1 < npts;
    float2* const conx = conx2 + buf * nk;
    // CONS of the two points by two threads of different warps, before the copy is awaited.
    if (tid == 0) cons2[buf].x = dia_cons(p, __ldg(kdmean + i0));
    if (tid == 32) cons2[buf].y = dia_cons(p, __ldg(kdmean + i1));
    const bool lost = !mbar_wait(bar, parity, err);
    parity ^= 1u;
    // 2a-2b. CON per frequency row and UE = A / CON, with the parametric tail up each column
    // from row NFR. The CTA's width is a whole number of rows, so a thread's bins are column r0
    // of rows q0, q0 + dq, ...: it forms each row's CON itself (the column-0 thread keeps it for
    // section 4), and one barrier follows instead of two. A bulk copy whose wait gave up ends
    // the CTA's work at that barrier, all its threads together.
    static_assert(dr == 0, "a whole number of rows per CTA");
    for (int row = q0; row < nk; row += dq) {
      const float w = wrow[row];
      const float2 cx = make_float2(w * stage[2 * nspec + row], w * stage[2 * nspec + nk + row]);
      if (r0 == 0) conx[row] = cx;
      const int isp = row * NTH + r0;
      const float2 v = make_float2(stage[isp] / cx.x, stage[nspec + isp] / cx.y);
      ue[isp + NTH] = v;
      if (row == nfr - 1) {
        float2 t = v;
        const float2 fh = dup2(p.fachfe);
        for (int r = nfr + 1; r <= p.nfrhgh; ++r) {
          t = mul2(t, fh);
          ue[r * NTH + r0] = t;
        }
      }
    }
    if (__syncthreads_or(lost)) break;

    const int pnext = pp + gridDim.x;
    if (tid == 0 && pnext < npairs) {
      const int j0 = first_of(pnext), j1 = second_of(pnext);
      tma_fetch_pair(bar, stage, a, cg, j0, j1, nspec, nk);
    }
    const float2 cons = cons2[buf];

    // 3. Interactions, BR rows unrolled.
    {
      float2 pa[4], pb[4], ma[4], mb[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int cp = c[j < 2 ? j : j + 2];  // c0 c1 c4 c5
        const int cm = c[j < 2 ? j + 2 : j + 4];  // c2 c3 c6 c7
        pa[j] = pp0[cp];
        pb[j] = pp0[NTH + cp];
        mb[j] = pm0[cm];
        ma[j] = pm0[NTH + cm];
      }
#pragma unroll
      for (int k = 0; k < BR; ++k) {
        {
          const int f = f0 + k;
          const float2 e00 = pe[k * NTH];
          const float2 ep1 = add2(add2(add2(mulS1(w0, pb[1]), mulS1(w1, pb[0])), mulS1(w2, pa[1])),
                                  mulS1(w3, pa[0]));
          const float2 em1 = add2(add2(add2(mulS1(w4, mb[3]), mulS1(w5, mb[2])), mulS1(w6, ma[3])),
                                  mulS1(w7, ma[2]));
          const float2 ep2 = add2(add2(add2(mulS1(w0, pb[3]), mulS1(w1, pb[2])), mulS1(w2, pa[3])),
                                  mulS1(w3, pa[2]));
          const float2 em2 = add2(add2(add2(mulS1(w4, mb[1]), mulS1(w5, mb[0])), mulS1(w6, ma[1])),
                                  mulS1(w7, ma[0]));
          const float2 ca = mul2(cons, dup2(afr[f - 1]));
          const float2 factor = mul2(ca, e00);
          const float2 sa1a = mulS(e00, add2(mulS1(dal1, ep1), mulS1(dal2, em1)));
          const float2 sa1b = sub2(sa1a, mulS1(dal3, mul2(ep1, em1)));
          const float2 sa2a = mulS(e00, add2(mulS1(dal1, ep2), mulS1(dal2, em2)));
          const float2 sa2b = sub2(sa2a, mulS1(dal3, mul2(ep2, em2)));
          po[k * NTH] = mul2(factor, sa1b);
          po[AS + k * NTH] = mul2(factor, sa2b);
          if (f <= nfr)
            pd[k * NTH] = add2(mulS(ca, add2(sa1a, sa1b)), mulS(ca, add2(sa2a, sa2b)));
          po[2 * AS + k * NTH] = mul2(factor, sub2(mulS1(dal1, e00), mulS1(dal3, em1)));
          po[3 * AS + k * NTH] = mul2(factor, sub2(mulS1(dal2, e00), mulS1(dal3, ep1)));
          po[4 * AS + k * NTH] = mul2(factor, sub2(mulS1(dal1, e00), mulS1(dal3, em2)));
          po[5 * AS + k * NTH] = mul2(factor, sub2(mulS1(dal2, e00), mulS1(dal3, ep2)));
          if (k + 1 < BR) {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              const int cp = c[j < 2 ? j : j + 2];
              const int cm = c[j < 2 ? j + 2 : j + 4];
              pa[j] = pb[j];
              mb[j] = ma[j];
              pb[j] = pp0[(k + 2) * NTH + cp];
              ma[j] = pm0[(k + 2) * NTH + cm];
            }
          }
        }
      }
    }
    __syncthreads();

    // 4. Source and diagonal terms, S then D, BR rows unrolled.
    {
      float2 l5[4], l6[4], h7[4], h8[4];
      float* const sp0 = s + static_cast<size_t>(i0) * nspec + (f0 - 1) * NTH + ith;
      float* const sp1 = s + static_cast<size_t>(i1) * nspec + (f0 - 1) * NTH + ith;
      float* const dp0 = d + static_cast<size_t>(i0) * nspec + (f0 - 1) * NTH + ith;
      float* const dp1 = d + static_cast<size_t>(i1) * nspec + (f0 - 1) * NTH + ith;
      const float2 m2 = dup2(-2.0f);
#pragma unroll
      for (int pass = 0; pass < 2; ++pass) {
        // pass 0: S from SA1 (lo c4 c5, hi c2 c3) and SA2 (lo c0 c1, hi c6 c7);
        // pass 1: D from DA1P/DA2P (lo) and DA1M/DA2M (hi).
        const int o1l = pass == 0 ? 0 : 2 * AS, o2l = pass == 0 ? AS : 4 * AS;
        const int o1h = pass == 0 ? 0 : 3 * AS, o2h = pass == 0 ? AS : 5 * AS;
        const float v0 = pass == 0 ? w0 : p.swg[0], v1 = pass == 0 ? w1 : p.swg[1];
        const float v2 = pass == 0 ? w2 : p.swg[2], v3 = pass == 0 ? w3 : p.swg[3];
        const float v4 = pass == 0 ? w4 : p.swg[4], v5 = pass == 0 ? w5 : p.swg[5];
        const float v6 = pass == 0 ? w6 : p.swg[6], v7 = pass == 0 ? w7 : p.swg[7];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int cl = j < 2 ? c[j + 4] : c[j - 2];  // c4 c5 | c0 c1
          const int ch = j < 2 ? c[j + 2] : c[j + 4];  // c2 c3 | c6 c7
          const int ol = j < 2 ? o1l : o2l, oh = j < 2 ? o1h : o2h;
          l6[j] = pl0[ol + cl];
          l5[j] = pl0[ol + NTH + cl];
          h7[j] = ph0[oh + ch];
          h8[j] = ph0[oh + NTH + ch];
        }
#pragma unroll
        for (int k = 0; k < BR; ++k) {
          const bool store = f0 + k <= nfr;
          {
            float2 t = pass == 0 ? mulS(m2, add2(po[k * NTH], po[AS + k * NTH]))
                                 : mulS(m2, pd[k * NTH]);
            t = add2(t, mulS1(v0, add2(l6[1], l6[3])));
            t = add2(t, mulS1(v1, add2(l6[0], l6[2])));
            t = add2(t, mulS1(v2, add2(l5[1], l5[3])));
            t = add2(t, mulS1(v3, add2(l5[0], l5[2])));
            t = add2(t, mulS1(v4, add2(h8[1], h8[3])));
            t = add2(t, mulS1(v5, add2(h8[0], h8[2])));
            t = add2(t, mulS1(v6, add2(h7[1], h7[3])));
            t = add2(t, mulS1(v7, add2(h7[0], h7[2])));
            if (pass == 0) {
              const float2 sv = mul2(conx[f0 + k - 1], t);
              if (store) __stcs(sp0 + k * NTH, sv.x);
              if (store && has1) __stcs(sp1 + k * NTH, sv.y);
            } else {
              if (store) __stcs(dp0 + k * NTH, t.x);
              if (store && has1) __stcs(dp1 + k * NTH, t.y);
            }
            if (k + 1 < BR) {
#pragma unroll
              for (int j = 0; j < 4; ++j) {
                const int cl = j < 2 ? c[j + 4] : c[j - 2];
                const int ch = j < 2 ? c[j + 2] : c[j + 4];
                const int ol = j < 2 ? o1l : o2l, oh = j < 2 ? o1h : o2h;
                l6[j] = l5[j];
                h7[j] = h8[j];
                l5[j] = pl0[ol + (k + 2) * NTH + cl];
                h8[j] = ph0[oh + (k + 2) * NTH + ch];
              }
            }
          }
        }
      }
    }
    // The next pair's barriers order its writes of UE and the arrays after this section 4.
  }
}

constexpr int kPairBlock = 288;
constexpr int kPairMinBlocks = 2;  // 2 CTAs of 288 threads per SM: at most 113 registers
constexpr int kPairStride = 1536;  // float2 slots per interaction array

constexpr int kBandBlock = 288;
constexpr int kTileMinBlocks = 2;  // 2 CTAs of 288 threads per SM: at most 113 registers
constexpr int kBandMinBlocks = 2;  // 2 CTAs of 288 threads per SM: at most 96 registers
int* g_band_err = nullptr;

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

namespace {
/// The interaction-array stride of the band kernel instance that fits these tables, or 0.
int band_stride(const Snl1Dev& p) {
  const int need = (p.nfrchg + 1) * p.nth;
  return need <= 1536 ? 1536 : (need <= 4096 ? 4096 : 0);
}
}  // namespace

namespace {
template <int NTH, int G, int BR>
size_t tile_smem(const Snl1Dev& p) {
  using S = TileShape<NTH, G, BR>;
  auto r4 = [](size_t n) { return (n + 3) & ~static_cast<size_t>(3); };
  const size_t floats = r4(static_cast<size_t>(p.nfrhgh + 1 + S::kPad) * NTH) + 6 * S::kAS +
                        static_cast<size_t>(S::kRows) * NTH + r4(2 * p.nk) + r4(p.nfrchg) +
                        r4(static_cast<size_t>(p.nspec + p.nk));
  return floats * sizeof(float) + 16;
}

/// Which tile instance fits these tables: 36 (8 bands of 5 rows) or 24 (12 bands of 3), or 0.
int tile_variant(const Snl1Dev& p) {
  if (p.ifrow == nullptr || p.af11_row == nullptr || p.ifrp < 0 || p.ifrm > 0) return 0;
  if (p.ifrp > 4 || -p.ifrm > 4) return 0;  // the zero rows below row 0
  if (p.nspec % 4 != 0 || p.nk % 4 != 0) return 0;  // bulk copies of A and CG
  if (p.nth == 36 && p.nfrchg <= 40) return 36;
  if (p.nth == 24 && p.nfrchg <= 36) return 24;
  return 0;
}
}  // namespace

bool snl1_tile_ok(const Snl1Dev& p) { return tile_variant(p) != 0; }

size_t snl1_band_smem(const Snl1Dev& p) {
  size_t floats = static_cast<size_t>(p.nfrhgh + 1) * p.nth + 6 * static_cast<size_t>(band_stride(p)) +
                  p.nspec + 2 * p.nk + p.nfrchg;
  floats = (floats + 3) & ~static_cast<size_t>(3);
  floats += (static_cast<size_t>(p.nspec + p.nk) + 3) & ~static_cast<size_t>(3);
  return floats * sizeof(float) + 16;  // + the mbarrier
}

bool snl1_band_ok(const Snl1Dev& p) {
  if (p.ifrow == nullptr || p.af11_row == nullptr) return false;  // no row-shift form
  if (p.nth > kBandBlock || p.ifrp < 0 || p.ifrm > 0 || band_stride(p) == 0) return false;
  return snl1_band_smem(p) <= 227 * 1024;
}

size_t snl1_pair_smem(const Snl1Dev& p) {
  size_t bytes = 8 * (static_cast<size_t>(p.nfrhgh + 1) * p.nth +
                      6 * static_cast<size_t>(kPairStride) + p.nspec + 2 * p.nk + 2) +
                 4 * static_cast<size_t>(p.nfrchg);
  bytes = (bytes + 15) & ~static_cast<size_t>(15);
  bytes += 4 * ((2 * static_cast<size_t>(p.nspec + p.nk) + 3) & ~static_cast<size_t>(3));
  return bytes + 16;  // + the mbarrier
}

bool snl1_pair_ok(const Snl1Dev& p) {
  if (p.ifrow == nullptr || p.af11_row == nullptr) return false;  // no row-shift form
  if (p.nth > kPairBlock || p.ifrp < 0 || p.ifrm > 0) return false;
  if ((p.nfrchg + 1) * p.nth > kPairStride) return false;
  if (p.nspec % 4 != 0 || p.nk % 4 != 0) return false;  // the bulk copies
  return snl1_pair_smem(p) <= 227 * 1024;
}

int snl1_take_error() {
  if (g_band_err == nullptr) return 0;
  int v = 0;
  WWB_CHECK(cudaMemcpy(&v, g_band_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (v != 0) WWB_CHECK(cudaMemset(g_band_err, 0, sizeof(int)));
  return v;
}

namespace {
template <int NTH, int G, int BR>
void launch_tile(const Snl1Dev& p, int npts, const float* a, const float* cg, const float* kd,
                 float* s, float* d, int* err, cudaStream_t stream) {
  static int per_sm = -1;
  static size_t cached = 0;
  const size_t smem = tile_smem<NTH, G, BR>(p);
  auto k = snl1_tile_kernel<NTH, G, BR, kTileMinBlocks>;
  if (per_sm < 0 || cached != smem) {
    WWB_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(smem)));
    int n = 0;
    WWB_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, NTH * G, smem));
    if (n < 1) throw CudaError(cudaErrorInvalidConfiguration, "snl1 tile occupancy");
    per_sm = n;
    cached = smem;
  }
  const long long resident = static_cast<long long>(per_sm) * runtime().sm_count;
  const int grid = static_cast<int>(npts < resident ? npts : resident);
  k<<<grid, NTH * G, smem, stream>>>(p, npts, a, cg, kd, s, d, err);
  WWB_CHECK(cudaGetLastError());
}

template <int AS, bool TMA>
void launch_band(const Snl1Dev& p, int npts, const float* a, const float* cg, const float* kd,
                 float* s, float* d, int* err, cudaStream_t stream) {
  static int per_sm = -1;
  static size_t cached = 0;
  const size_t smem = snl1_band_smem(p);
  auto k = snl1_band_kernel<kBandBlock, kBandMinBlocks, AS, TMA>;
  if (per_sm < 0 || cached != smem) {
    WWB_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(smem)));
    int n = 0;
    WWB_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, kBandBlock, smem));
    if (n < 1) throw CudaError(cudaErrorInvalidConfiguration, "snl1 band occupancy");
    per_sm = n;
    cached = smem;
  }
  const long long resident = static_cast<long long>(per_sm) * runtime().sm_count;
  const int grid = static_cast<int>(npts < resident ? npts : resident);
  k<<<grid, kBandBlock, smem, stream>>>(p, npts, a, cg, kd, s, d, err, nullptr, nullptr);
  WWB_CHECK(cudaGetLastError());
}

// The pair-tile instance: 36 directions, 8 bands of 5 rows, zero rows 3 below UE and 2 below the
// interaction arrays.
using PairTile36 = PairTileShape<36, 8, 5, 3, 2>;

/// Whether the 36-direction pair-tile instance fits these tables (every row it reads within its
/// padded matrices, the bulk copies 16-byte sized).
bool pairtile36_ok(const Snl1Dev& p) {
  if (p.ifrow == nullptr || p.af11_row == nullptr || p.nth != 36) return false;
  if (p.nspec % 4 != 0 || p.nk % 4 != 0) return false;
  if (p.ifrp < 0 || p.ifrm > 0 || p.ifrp > 2 || -p.ifrm > 3) return false;
  // Section 3 fills the 8 x 5 rows exactly; section 4's NFR rows fit in them.
  if (p.nfr > 40 || p.nfrchg != 40 || p.nfrchg + p.ifrp + 1 > p.nfrhgh) return false;
  if (p.nspec > PairTile36::kDcs) return false;
  if (p.nfrhgh > 40 + 2 + 1 || p.nfr - p.ifrm + 1 > p.nfrchg) return false;
  return true;
}

size_t pairtile36_smem(const Snl1Dev& p) {
  using S = PairTile36;
  size_t bytes = 8 * (static_cast<size_t>(S::kRowsU) * 36 + 6 * static_cast<size_t>(S::kAS) +
                      S::kDcs + 2 * p.nk + 2) +
                 4 * static_cast<size_t>(p.nfrchg + p.nk);
  bytes = (bytes + 15) & ~static_cast<size_t>(15);
  bytes += 4 * ((2 * static_cast<size_t>(p.nspec + p.nk) + 3) & ~static_cast<size_t>(3));
  return bytes + 16;  // + the mbarrier
}

template <bool LIST>
void launch_pairtile36(const Snl1Dev& p, int capacity, const int* pidx, const int* pcount,
                       const float* a, const float* cg, const float* kd, float* s, float* d,
                       int* err, cudaStream_t stream) {
  static int per_sm = -1;
  static size_t cached = 0;
  const size_t smem = pairtile36_smem(p);
  auto k = snl1_pairtile_kernel<36, 8, 5, 3, 2, LIST>;
  if (per_sm < 0 || cached != smem) {
    WWB_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(smem)));
    int n = 0;
    WWB_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, PairTile36::kBlock, smem));
    if (n < 1) throw CudaError(cudaErrorInvalidConfiguration, "snl1 pair-tile occupancy");
    per_sm = n;
    cached = smem;
  }
  const long long pairs = (static_cast<long long>(capacity) + 1) / 2;
  const long long resident = static_cast<long long>(per_sm) * runtime().sm_count;
  const int grid = static_cast<int>(pairs < resident ? pairs : resident);
  k<<<grid, PairTile36::kBlock, smem, stream>>>(p, capacity, a, cg, kd, s, d, err, pidx, pcount);
  WWB_CHECK(cudaGetLastError());
}

/// The pair kernel: its 36-direction tile instance where that fits (unless `general`), else
/// its general form.
template <bool LIST>
void launch_pair(const Snl1Dev& p, int capacity, const int* pidx, const int* pcount,
                 const float* a, const float* cg, const float* kd, float* s, float* d, int* err,
                 cudaStream_t stream, bool general = false) {
  if (pairtile36_ok(p) && !general)
    return launch_pairtile36<LIST>(p, capacity, pidx, pcount, a, cg, kd, s, d, err, stream);
  static int per_sm = -1;
  static size_t cached = 0;
  const size_t smem = snl1_pair_smem(p);
  auto k = snl1_pair_kernel<kPairBlock, kPairMinBlocks, kPairStride, LIST>;
  if (per_sm < 0 || cached != smem) {
    WWB_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(smem)));
    int n = 0;
    WWB_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, kPairBlock, smem));
    if (n < 1) throw CudaError(cudaErrorInvalidConfiguration, "snl1 pair occupancy");
    per_sm = n;
    cached = smem;
  }
  const long long pairs = (static_cast<long long>(capacity) + 1) / 2;
  const long long resident = static_cast<long long>(per_sm) * runtime().sm_count;
  const int grid = static_cast<int>(pairs < resident ? pairs : resident);
  k<<<grid, kPairBlock, smem, stream>>>(p, capacity, a, cg, kd, s, d, err, pidx, pcount);
  WWB_CHECK(cudaGetLastError());
}

/// The error flag of the band and tile kernels' bulk-copy waits (allocated on first use).
int* band_err_flag() {
  if (g_band_err == nullptr) {
    WWB_CHECK(cudaMalloc(&g_band_err, sizeof(int)));
    WWB_CHECK(cudaMemset(g_band_err, 0, sizeof(int)));
  }
  return g_band_err;
}

/// Launches `kernel`; the band and tile kernels report a bulk-copy wait that gave up in `err`,
/// or in the shared flag band_err_flag() when `err` is null.
void launch_dispatch(int kernel, const Snl1Dev& p, int npts, const float* a, const float* cg,
                     const float* kdmean, float* s, float* d, int* err, cudaStream_t stream);
}  // namespace

void launch_snl1(int kernel, const Snl1Dev& p, int npts, const float* a, const float* cg,
                 const float* kdmean, float* s, float* d, cudaStream_t stream) {
  launch_dispatch(kernel, p, npts, a, cg, kdmean, s, d, nullptr, stream);
}

namespace {
void launch_dispatch(int kernel, const Snl1Dev& p, int npts, const float* a, const float* cg,
                     const float* kdmean, float* s, float* d, int* err, cudaStream_t stream) {
  if (npts <= 0) return;
  if (kernel == kSnl1Tile || kernel == kSnl1Band || kernel == kSnl1Pair ||
      kernel == kSnl1PairGeneral) {
    if (err == nullptr) err = band_err_flag();
  }
  const bool aligned = (reinterpret_cast<uintptr_t>(a) & 15u) == 0 &&
                       (reinterpret_cast<uintptr_t>(cg) & 15u) == 0;
  if (kernel == kSnl1Pair || kernel == kSnl1PairGeneral) {
    if (aligned && snl1_pair_ok(p))
      return launch_pair<false>(p, npts, nullptr, nullptr, a, cg, kdmean, s, d, err, stream,
                                kernel == kSnl1PairGeneral);
    kernel = kSnl1Band;  // caller arrays not 16-byte aligned: the band kernel reads them directly
  }
  if (kernel == kSnl1Tile) {
    const int v = tile_variant(p);
    if (v == 36 && aligned) return launch_tile<36, 8, 5>(p, npts, a, cg, kdmean, s, d, err, stream);
    if (v == 24 && aligned) return launch_tile<24, 12, 3>(p, npts, a, cg, kdmean, s, d, err, stream);
    kernel = kSnl1Band;  // caller arrays not 16-byte aligned: the band kernel reads them directly
  }
  if (kernel == kSnl1Band) {
    // The bulk copies need 16-byte aligned sources and sizes: NSPEC and NK multiples of 4.
    const bool tma = p.nspec % 4 == 0 && p.nk % 4 == 0 && aligned;
    if (band_stride(p) == 1536) {
      if (tma) launch_band<1536, true>(p, npts, a, cg, kdmean, s, d, err, stream);
      else launch_band<1536, false>(p, npts, a, cg, kdmean, s, d, err, stream);
    } else {
      if (tma) launch_band<4096, true>(p, npts, a, cg, kdmean, s, d, err, stream);
      else launch_band<4096, false>(p, npts, a, cg, kdmean, s, d, err, stream);
    }
  } else if (kernel == kSnl1RowShift) {
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
}  // namespace

// ------------------------------------------------------------------------------------------
// Storage of the entry that allocates nothing (ww_snl1_noalloc): one file-scope device array
// for the staged A, CG, KDMEAN, S and D, and the bulk-copy error flag of its launches. Both
// exist once per device for the whole process, so calls that overlap in time (two host
// threads, or work still in flight on another stream) race on them.
constexpr size_t kStaticScratchFloats = static_cast<size_t>(8) << 20;  // 32 MiB
static __device__ __align__(256) float g_static_scratch[kStaticScratchFloats];
static __device__ int g_static_err;

namespace {
constexpr int kStaticMaxDevices = 64;
Snl1StaticScratch g_static_dev[kStaticMaxDevices];  // resolved addresses, per device
}  // namespace

Snl1StaticScratch snl1_static_scratch() {
  int dev = 0;
  WWB_CHECK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kStaticMaxDevices)
    throw CudaError(cudaErrorInvalidDevice, "snl1 static scratch: device ordinal out of range");
  Snl1StaticScratch& e = g_static_dev[dev];
  if (e.base == nullptr) {
    // Set-up, once per device with that device current: resolve the arrays' addresses.
    void* base = nullptr;
    void* err = nullptr;
    cudaError_t rc = cudaGetSymbolAddress(&base, g_static_scratch);
    if (rc != cudaSuccess) throw CudaError(rc, "snl1 static scratch: cudaGetSymbolAddress");
    rc = cudaGetSymbolAddress(&err, g_static_err);
    if (rc != cudaSuccess) throw CudaError(rc, "snl1 static error flag: cudaGetSymbolAddress");
    e.floats = kStaticScratchFloats;
    e.err = static_cast<int*>(err);
    e.base = static_cast<float*>(base);
  }
  return e;
}

void launch_snl1_err(int kernel, const Snl1Dev& p, int npts, const float* a, const float* cg,
                     const float* kdmean, float* s, float* d, int* err, cudaStream_t stream) {
  if (err == nullptr) throw CudaError(cudaErrorInvalidValue, "launch_snl1_err: null error flag");
  launch_dispatch(kernel, p, npts, a, cg, kdmean, s, d, err, stream);
}

namespace {
template <int AS, bool TMA>
void launch_band_list(const Snl1Dev& p, int capacity, const int* pidx, const int* pcount,
                      const float* a, const float* cg, const float* kd, float* s, float* d,
                      int* err, cudaStream_t stream) {
  static int per_sm = -1;
  static size_t cached = 0;
  const size_t smem = snl1_band_smem(p);
  auto k = snl1_band_kernel<kBandBlock, kBandMinBlocks, AS, TMA, true>;
  if (per_sm < 0 || cached != smem) {
    WWB_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(smem)));
    int n = 0;
    WWB_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, kBandBlock, smem));
    if (n < 1) throw CudaError(cudaErrorInvalidConfiguration, "snl1 band occupancy");
    per_sm = n;
    cached = smem;
  }
  const long long resident = static_cast<long long>(per_sm) * runtime().sm_count;
  const int grid = static_cast<int>(capacity < resident ? capacity : resident);
  k<<<grid, kBandBlock, smem, stream>>>(p, capacity, a, cg, kd, s, d, err, pidx, pcount);
  WWB_CHECK(cudaGetLastError());
}
}  // namespace

bool launch_snl1_list(const Snl1Dev& p, int capacity, const int* pidx, const int* pcount,
                      const float* a, const float* cg, const float* kdmean, float* s, float* d,
                      int* err, cudaStream_t stream) {
  if (capacity <= 0) return true;
  if (!snl1_band_ok(p)) return false;
  if (err == nullptr) err = band_err_flag();
  const bool aligned = (reinterpret_cast<uintptr_t>(a) & 15u) == 0 &&
                       (reinterpret_cast<uintptr_t>(cg) & 15u) == 0;
  if (aligned && snl1_pair_ok(p)) {
    launch_pair<true>(p, capacity, pidx, pcount, a, cg, kdmean, s, d, err, stream);
    return true;
  }
  const bool tma = p.nspec % 4 == 0 && p.nk % 4 == 0 && aligned;
  if (band_stride(p) == 1536) {
    if (tma) launch_band_list<1536, true>(p, capacity, pidx, pcount, a, cg, kdmean, s, d, err, stream);
    else launch_band_list<1536, false>(p, capacity, pidx, pcount, a, cg, kdmean, s, d, err, stream);
  } else {
    if (tma) launch_band_list<4096, true>(p, capacity, pidx, pcount, a, cg, kdmean, s, d, err, stream);
    else launch_band_list<4096, false>(p, capacity, pidx, pcount, a, cg, kdmean, s, d, err, stream);
  }
  return true;
}

}  // namespace wwb
