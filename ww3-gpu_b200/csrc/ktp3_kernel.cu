// ww3-gpu_b200/csrc/ktp3_kernel.cu
// W3KTP3 with W3QCK1/W3QCK2 for sm_100a: one CTA per sea point, the rotated (NK+2) x (NTH+3)
// work spectrum VQ and every work array of the point in shared memory.
//
// The reference runs each point serially (kokkos/src/ww_kokkos/prop_ktp3.hpp:132-353). Inside
// a point every loop here is data-parallel: each element of DSDD, VQ, VCFLT, DB/DM, CFLK and FLA
// is written by one thread from inputs no thread modifies in the same phase, and the phases
// are separated by CTA barriers, so the arithmetic of each element is the reference's,
// operation for operation (-fmad=false). The two reductions, CFLTHMAX and CFLKMAX, are maxima
// of absolute values; for inputs without NaN any association gives the reference's bits
// (prop_ktp3.hpp:281-309 groups lanes only as its vectorised -O3 build did, which matters for
// NaN alone).
//
// W3QCK1 (prop_qck1.hpp) is called with CLOSE true (periodic in direction): its closure copies
// are per row IY, so one thread takes a whole row in statement order. W3QCK2 (prop_qck2.hpp) is
// called with CLOSE false.
#include "ktp3_kernel.cuh"

#include <climits>

#include "wwb_common.hpp"

namespace wwb {
namespace {

constexpr int kKtp3Block = 256;

__device__ __forceinline__ float max_r(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float min_r(float a, float b) { return a < b ? a : b; }
/// INT(x) of a REAL as gfortran's cvttss2si: truncation, INT_MIN for NaN or out of range.
__device__ __forceinline__ int fint(float x) {
  return (x > -2147483904.0f && x < 2147483648.0f) ? static_cast<int>(x) : INT_MIN;
}

struct Work {
  float *va, *vq, *dsdd, *frk, *frg, *fkc, *db, *dm, *vcflt, *cflk, *fla, *cg, *wn, *red;
};

__device__ Work carve(float* base, int nk, int nth, int nspec) {
  const int nk2 = nk + 2;
  Work w;
  w.va = base;
  w.vq = w.va + nspec;
  w.dsdd = w.vq + nk2 * (nth + 3);
  w.frk = w.dsdd + nk2;
  w.frg = w.frk + nk;
  w.fkc = w.frg + nk;
  w.db = w.fkc + nth;
  w.dm = w.db + nk2 * (nth + 1);
  w.vcflt = w.dm + nk2 * (nth + 2);
  w.cflk = w.vcflt + nk2 * (nth + 1);
  w.fla = w.cflk + nk2 * (nth + 1);
  w.cg = w.fla + nk2 * (nth + 1);
  w.wn = w.cg + nk2;
  w.red = w.wn + nk2;
  return w;
}

/// max_r-reduction of one value per thread over the CTA (result in every thread).
__device__ float block_max(float v, float* red) {
  for (int o = 16; o > 0; o >>= 1) v = max_r(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) red[warp] = v;
  __syncthreads();
  float r = red[0];
  for (int i = 1; i < kKtp3Block / 32; ++i) r = max_r(r, red[i]);
  __syncthreads();
  return r;
}

/// W3QCK1 with CLOSE true (w3uqckmd.F90:281-426 as prop_qck1.hpp states it), CTA-cooperative.
__device__ void qck1_cta(int mx, int my, int nx, int ny, float* cfll, float* q, int inc,
                         const int* __restrict__ mapact, int nact,
                         const int* __restrict__ mapbou, int nb0, int nb1, int nb2, float* fla) {
  const int qoff = my - 1, foff = my - 1;
  const int tid = threadIdx.x;
  for (int i = tid; i < my * (mx + 1); i += kKtp3Block) fla[i] = 0.0f;
  const int iad00 = -my, iad02 = my, iadn0 = iad00 + my * nx, iadn1 = my * nx,
            iadn2 = iad02 + my * nx;
  for (int iy = 1 + tid; iy <= ny; iy += kKtp3Block) {  // closure part 1, a row per thread
    q[iy + iad00 + qoff] = q[iy + iadn0 + qoff];
    q[iy + iadn1 + qoff] = q[iy + qoff];
    q[iy + iadn2 + qoff] = q[iy + iad02 + qoff];
    cfll[iy + iadn1 - 1] = cfll[iy - 1];
  }
  __syncthreads();
  for (int ip = 1 + tid; ip <= nb2; ip += kKtp3Block) {
    const int ixy = __ldg(mapbou + ip - 1);
    if (ip <= nb0) {  // central points
      const float cfl = (cfll[ixy + inc - 1] + cfll[ixy - 1]) * 0.5f;
      const float s = copysignf(1.1f, cfl);
      const int ixyc = ixy - inc * fint(min_r(s, 0.0f));
      const float c2 = cfl * cfl;
      const float t2 = (1.0f - cfl) * q[ixy + inc + qoff];
      const float t4 = (cfl + 1.0f) * q[ixy + qoff];
      const float t6 = (t4 + t2) * 0.5f;
      const float t8 = (1.0f - c2) / 6.0f;
      const float qixyc = q[ixyc + qoff];
      const float t9 = qixyc * 2.0f;
      const float t11 = q[ixyc + inc + qoff] + (q[ixyc - inc + qoff] - t9);
      const float qb = t6 - t11 * t8;
      const int ixyu = ixyc - inc * fint(s);
      const int ixyd = 2 * ixyc - ixyu;
      const float qixyu = q[ixyu + qoff];
      const float dq = q[ixyd + qoff] - qixyu;
      const float dqnz = copysignf(max_r(fabsf(dq), 1.e-15f), dq);
      const float qcn = min_r(max_r((qixyc - qixyu) / dqnz, -0.1f), 1.1f);
      const float qbn0 = max_r((qb - qixyu) / dqnz, qcn);
      const float t13 = min_r(qcn / max_r(fabsf(cfl), 1.e-10f), 1.0f);
      const float qbn = min_r(qbn0, t13);
      const float qbr = qbn * dq + qixyu;
      const float cfac = static_cast<float>(fint(fabsf(qcn - 0.5f) * 2.0f));
      const float qb2 = cfac * qixyc + (1.0f - cfac) * qbr;
      fla[ixy + foff] = qb2 * cfl;
    } else {  // boundary above (CFL at IXY) or below (CFL at IXY+INC)
      const float cfl = ip <= nb1 ? cfll[ixy - 1] : cfll[ixy + inc - 1];
      const float s = copysignf(1.1f, cfl);
      const int ixyc = ixy - inc * fint(min_r(s, 0.0f));
      fla[ixy + foff] = q[ixyc + qoff] * cfl;
    }
  }
  __syncthreads();
  for (int iy = 1 + tid; iy <= ny; iy += kKtp3Block)  // closure part 2
    fla[iy + iad00 + foff] = fla[iy + iadn0 + foff];
  __syncthreads();
  for (int ip = 1 + tid; ip <= nact; ip += kKtp3Block) {
    const int ixy = __ldg(mapact + ip - 1);
    const float u = (q[ixy + qoff] + fla[ixy - inc + foff]) - fla[ixy + foff];
    q[ixy + qoff] = max_r(u, 0.0f);
  }
  __syncthreads();
}

/// W3QCK2 with CLOSE false (w3uqckmd.F90:680-841 as prop_qck2.hpp states it), CTA-cooperative.
__device__ void qck2_cta(int mx, int my, float* velo, float dt, const float* dx1,
                         const float* dx2, float* q, int inc, const int* __restrict__ mapact,
                         int nact, const int* __restrict__ mapbou, int nb0, int nb1, int nb2,
                         float* fla) {
  const int qoff = my - 1;
  const int tid = threadIdx.x;
  for (int i = tid; i < my * (mx + 1); i += kKtp3Block) fla[i] = 0.0f;
  __syncthreads();
  for (int ip = 1 + tid; ip <= nb2; ip += kKtp3Block) {
    const int ixy = __ldg(mapbou + ip - 1);
    if (ip <= nb0) {
      const float vel = (velo[ixy + inc - 1] + velo[ixy - 1]) * 0.5f;
      const float dx2ixy = dx2[ixy + qoff];
      const float cfl = (dt * vel) / dx2ixy;
      const float s = copysignf(1.1f, cfl);
      const int ixyc = ixy - inc * fint(min_r(s, 0.0f));
      const float d2 = dx2ixy * dx2ixy;
      const float c2 = cfl * cfl;
      const float t2 = q[ixy + inc + qoff] * (1.0f - cfl);
      const float t4 = q[ixy + qoff] * (cfl + 1.0f);
      const float t6 = (t4 + t2) * 0.5f;
      const float t8 = ((1.0f - c2) * (d2 / dx1[ixyc - 1])) / 6.0f;
      const float qixyc = q[ixyc + qoff];
      const float u1 = (q[ixyc + inc + qoff] - qixyc) / dx2[ixyc + qoff];
      const float u2 = (qixyc - q[ixyc - inc + qoff]) / dx2[ixyc - inc + qoff];
      const float qb = t6 - (u1 - u2) * t8;
      const int ixyu = ixyc - inc * fint(s);
      const int ixyd = 2 * ixyc - ixyu;
      const float qixyu = q[ixyu + qoff];
      const float dq = q[ixyd + qoff] - qixyu;
      const float dqnz = copysignf(max_r(fabsf(dq), 1.e-15f), dq);
      const float qcn = min_r(max_r((qixyc - qixyu) / dqnz, -0.1f), 1.1f);
      const float qbn0 = max_r((qb - qixyu) / dqnz, qcn);
      const float t13 = min_r(qcn / max_r(fabsf(cfl), 1.e-10f), 1.0f);
      const float qbn = min_r(qbn0, t13);
      const float qbr = qbn * dq + qixyu;
      const float cfac = static_cast<float>(fint(fabsf(qcn - 0.5f) * 2.0f));
      const float qb2 = cfac * qixyc + (1.0f - cfac) * qbr;
      fla[ixy + qoff] = qb2 * vel;
    } else {
      const float vel = ip <= nb1 ? velo[ixy - 1] : velo[ixy + inc - 1];
      const float s = copysignf(1.1f, vel);
      const int ixyc = ixy - inc * fint(min_r(s, 0.0f));
      fla[ixy + qoff] = q[ixyc + qoff] * vel;
    }
  }
  __syncthreads();
  for (int ip = 1 + tid; ip <= nact; ip += kKtp3Block) {
    const int ixy = __ldg(mapact + ip - 1);
    const float f = dt / dx1[ixy - 1];
    const float u = q[ixy + qoff] + f * (fla[ixy - inc + qoff] - fla[ixy + qoff]);
    q[ixy + qoff] = max_r(u, 0.0f);
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kKtp3Block) ktp3_kernel(
    const Ktp3Dev p, const int itstep, const int ntimes, const float facth, const float fack,
    const int npts, const int* __restrict__ jsea, const int* __restrict__ isea,
    const float* __restrict__ pscal, const float* __restrict__ cgg,
    const float* __restrict__ wng, float* __restrict__ va, float* __restrict__ cflth_out,
    float* __restrict__ cflk_out) {
  extern __shared__ __align__(16) float smem[];
  const int nk = p.nk, nth = p.nth, nspec = p.nspec, nk2 = p.nk2;
  const Work w = carve(smem, nk, nth, nspec);
  const int tid = threadIdx.x;
  const int vqoff = nk2 - 1;  // VQ(I) = vq[I + NK2 - 1], lower bound 1-NK2
  const int* __restrict__ mapth2 = p.mapth2;

  for (int j = blockIdx.x; j < npts; j += gridDim.x) {
    const int js = __ldg(jsea + j), is = __ldg(isea + j);
    const float* ps = pscal + static_cast<size_t>(10) * j;
    const float cthg0 = __ldg(ps + 0), dw = __ldg(ps + 1), dddx = __ldg(ps + 2),
                dddy = __ldg(ps + 3), cx = __ldg(ps + 4), cy = __ldg(ps + 5),
                dcxdx = __ldg(ps + 6), dcxdy = __ldg(ps + 7), dcydx = __ldg(ps + 8),
                dcydy = __ldg(ps + 9);
    float* const vcol = va + static_cast<size_t>(js) * nspec;
    for (int i = tid; i < nspec; i += kKtp3Block) w.va[i] = vcol[i];
    for (int i = tid; i < nk2; i += kKtp3Block) {
      w.cg[i] = __ldg(cgg + static_cast<size_t>(is) * nk2 + i);
      w.wn[i] = __ldg(wng + static_cast<size_t>(is) * nk2 + i);
    }
    float acc_th = 0.0f, acc_k = 0.0f;
    for (int t = 0; t < ntimes; ++t) {
      __syncthreads();  // previous point/pass done with every array
      // 1.a, 2.a: depth, the zero fills, DSDD.
      const float depth = max_r(p.dmin, dw);
      for (int i = tid; i < nk2 * (nth + 3); i += kKtp3Block) w.vq[i] = 0.0f;
      if (p.flcth)
        for (int i = tid; i < nk2 * (nth + 1); i += kKtp3Block) w.vcflt[i] = 0.0f;
      if (p.flck)
        for (int i = tid; i < nk2 * (nth + 1); i += kKtp3Block) w.cflk[i] = 0.0f;
      for (int ik = tid; ik <= nk + 1; ik += kKtp3Block) {
        if (w.wn[ik] * depth < 5.0f) {
          const float tt = w.wn[ik] * w.cg[ik] - __ldg(p.sig + ik) * 0.5f;
          w.dsdd[ik] = max_r(tt, 0.0f) / depth;
        } else {
          w.dsdd[ik] = 0.0f;
        }
      }
      __syncthreads();
      // 2.b: scatter into the rotated space; 3.a: FRK, FRG.
      for (int isp = tid; isp < nspec; isp += kKtp3Block)
        w.vq[__ldg(mapth2 + isp) + vqoff] = w.va[isp];
      if (p.flcth) {
        const float fdg = cthg0 * facth;
        for (int ik = 1 + tid; ik <= nk; ik += kKtp3Block) {
          w.frk[ik - 1] = (facth * w.dsdd[ik]) / w.wn[ik];
          w.frg[ik - 1] = fdg * w.cg[ik];
        }
        // 3.b: current refraction scattered through MAPTH2 (else VCFLT stays zero).
        if (p.flcur) {
          const float dcyx = dcydx * facth;
          const float dcxxyy = (dcxdx - dcydy) * facth;
          const float dcxy = dcxdy * facth;
          for (int isp = tid; isp < nspec; isp += kKtp3Block)
            w.vcflt[__ldg(mapth2 + isp) - 1] =
                ((__ldg(p.es2 + isp) * dcyx) + (__ldg(p.esc + isp) * dcxxyy)) -
                (__ldg(p.ec2 + isp) * dcxy);
        }
      }
      if (p.flck) {
        // 4.a: FKC over the first NTH trig entries; 4.b: band widths in column 1.
        const float dcxx = -dcxdx;
        const float dcxyyx = -(dcxdy + dcydx);
        const float dcyy = -dcydy;
        for (int ith = tid; ith < nth; ith += kKtp3Block)
          w.fkc[ith] = ((__ldg(p.ec2 + ith) * dcxx) + (__ldg(p.esc + ith) * dcxyyx)) +
                       (__ldg(p.es2 + ith) * dcyy);
        for (int ik = tid; ik <= nk + 1; ik += kKtp3Block) {
          w.db[ik] = __ldg(p.dsip + ik) / w.cg[ik];
          w.dm[ik + nk2] = ik <= nk ? w.wn[ik + 1] - w.wn[ik] : 0.0f;
        }
      }
      __syncthreads();
      // 3.c: total velocity in direction, the CTMAX limiter, CFLTHMAX.
      if (p.flcth) {
        float acc = 0.0f;
        for (int isp = tid; isp < nspec; isp += kKtp3Block) {
          const int m2 = __ldg(mapth2 + isp);
          const int mw = __ldg(p.mapwn + isp);
          const float ec = __ldg(p.ecos + isp), es = __ldg(p.esin + isp);
          const float v = (w.vcflt[m2 - 1] + w.frg[mw - 1] * ec) +
                          w.frk[mw - 1] * ((es * dddx) - (ec * dddy));
          const float av = fabsf(v);
          acc = max_r(acc, av);
          w.vcflt[m2 - 1] = copysignf(min_r(av, p.ctmax), v);
        }
        acc_th = block_max(acc, w.red);
      }
      // 4.b: copy column 1 of DB and DM to columns 2..NTH; 4.c: CFLK and CFLKMAX.
      if (p.flck) {
        for (int i = tid; i < (nth - 1) * nk2; i += kKtp3Block) {
          const int ith = 2 + i / nk2, ik = 1 + i % nk2;
          w.db[(ik - 1) + (ith - 1) * nk2] = w.db[ik - 1];
          w.dm[(ik - 1) + ith * nk2] = w.dm[(ik - 1) + nk2];
        }
        const float fkd = (cx * dddx) + (cy * dddy);
        float acc = 0.0f;
        for (int i = tid; i < nk2 * nth; i += kKtp3Block) {
          const int ik = i % nk2, ith = 1 + i / nk2;
          const float fkd0 = (fkd / w.cg[ik]) * w.dsdd[ik];
          const float velfac = fack / w.db[ik];
          const float v = ((w.wn[ik] * w.fkc[ith - 1]) + fkd0) * velfac;
          w.cflk[ik + (ith - 1) * nk2] = copysignf(min_r(p.ctmax, fabsf(v)), v) / velfac;
          acc = max_r(acc, fabsf(v));
        }
        acc_k = block_max(acc, w.red);
      }
      __syncthreads();
      // 5. Propagate: the k pass first on an even ITSTEP, the theta pass first on an odd one.
      for (int pass = 0; pass < 2; ++pass) {
        const bool kpass = (itstep % 2 == 0) == (pass == 0);
        if (kpass && p.flck) {
          for (int ith = 1 + tid; ith <= nth; ith += kKtp3Block)
            w.vq[nk + 2 + (ith - 1) * nk2 + vqoff] =
                p.fachfa * w.vq[nk + 1 + (ith - 1) * nk2 + vqoff];
          __syncthreads();
          qck2_cta(nth, nk2, w.cflk, fack, w.db, w.dm, w.vq, 1, mapth2, nspec, p.mapwn2,
                   nspec - nth, nspec, nspec + nth, w.fla);
        } else if (!kpass && p.flcth) {
          qck1_cta(nth, nk2, nth, nk2, w.vcflt, w.vq, nk2, mapth2, nspec, mapth2, nspec, nspec,
                   nspec, w.fla);
        }
      }
      // 6. Store back from the rotated space.
      for (int isp = tid; isp < nspec; isp += kKtp3Block)
        w.va[isp] = w.vq[__ldg(mapth2 + isp) + vqoff];
    }
    __syncthreads();
    for (int i = tid; i < nspec; i += kKtp3Block) vcol[i] = w.va[i];
    if (tid == 0) {
      cflth_out[js - 1] = acc_th;
      cflk_out[js - 1] = acc_k;
    }
  }
}

}  // namespace

size_t ktp3_smem(const Ktp3Dev& p) {
  const size_t nk2 = p.nk2, nth = p.nth;
  return sizeof(float) * (p.nspec + nk2 * (nth + 3) + nk2 + 2 * p.nk + nth + nk2 * (nth + 1) +
                          nk2 * (nth + 2) + 3 * nk2 * (nth + 1) + 2 * nk2 + 32);
}

void launch_ktp3(const Ktp3Dev& p, int itstep, int ntimes, float facth, float fack, int npts,
                 const int* jsea, const int* isea, const float* pscal, const float* cg,
                 const float* wn, float* va, float* cflth, float* cflk, cudaStream_t stream) {
  if (npts <= 0 || ntimes <= 0) return;
  const size_t smem = ktp3_smem(p);
  WWB_CHECK(cudaFuncSetAttribute(ktp3_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem)));
  int per_sm = 0;
  WWB_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ktp3_kernel, kKtp3Block, smem));
  if (per_sm < 1) throw CudaError(cudaErrorInvalidConfiguration, "ktp3 occupancy");
  const long long resident = static_cast<long long>(per_sm) * runtime().sm_count;
  const int grid = static_cast<int>(npts < resident ? npts : resident);
  ktp3_kernel<<<grid, kKtp3Block, smem, stream>>>(p, itstep, ntimes, facth, fack, npts, jsea,
                                                   isea, pscal, cg, wn, va, cflth, cflk);
  WWB_CHECK(cudaGetLastError());
}

}  // namespace wwb
