// ww3-gpu_b200/csrc/wave_kernel.cu
// W3WAVE's per-step support routines on sm_100a (see wave_kernel.cuh). Each is a loop over sea
// points or grid cells in which an iteration reads inputs and writes only its own outputs, so
// one thread per point or cell gives the Fortran loop's bits; the expressions keep the
// reference's operand order, MAX keeps the build's maxss operand order, and the libm calls are
// the glibc-equal device functions (atan2f, sincosf, tanhf, coshf, sinhf). MOD(a, TPI) is fmodf,
// which is exact, as the Fortran's fprem loop is.
//
// Reference: ww3-gpu kokkos/src/ww_kokkos/wave_gath_scat.hpp:48-93 (W3GATH, W3SCAT),
// updt_uwnd.hpp:70-217 (W3UWND under WNT1 and RWND), updt_dzxy.hpp:60-224 (W3DZXY),
// disp_distab.hpp:77-185 (WAVNU2 and DISTAB), prop_cflxy.hpp:25-135 (W3CFLXY).
#include "wave_kernel.cuh"

#include "libm_dev.cuh"
#include "wavnu2_dev.cuh"
#include "wwb_common.hpp"

namespace wwb {
namespace {

// constants.F90's PI as REAL and TPI = 2*PI (an exact doubling). GRAV is disp::kGravD.
constexpr float kPi = static_cast<float>(3.141592653589793);
constexpr float kTpi = 2.0f * kPi;

/// Fortran MAX of two REALs as the build's maxss: a NaN or a tie gives the first operand.
__device__ __forceinline__ float fmax2(float a, float b) { return (b > a) ? b : a; }
__device__ __forceinline__ float mod_tpi(float a) { return fmodf(a, kTpi); }

int blocks(long long n, int per) {
  const long long b = (n + per - 1) / per;
  return static_cast<int>(b < 1 ? 1 : (b > 65535 ? 65535 : b));
}

#define WWB_GRID_LOOP(i, n)                                                    \
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < (n); \
       i += static_cast<long long>(gridDim.x) * blockDim.x)

// ------------------------------------------------------------------------------ W3GATH / W3SCAT
__global__ void gath_kernel(int nsea, int ny, const float* __restrict__ row,
                            const int* __restrict__ ixy, float* field) {
  WWB_GRID_LOOP(i, nsea) {
    const long long c = ixy[i];
    field[c - (1 - static_cast<long long>(ny))] = row[i + 1];
  }
}

__global__ void scat_kernel(int nsea, int ny, const int* __restrict__ mapsta,
                            const float* __restrict__ field, const int* __restrict__ ixy,
                            float* row) {
  WWB_GRID_LOOP(i, nsea) {
    const long long c = ixy[i];
    if (mapsta[c - 1] != 0) row[i + 1] = field[c - (1 - static_cast<long long>(ny))];
  }
}

// ------------------------------------------------------------------------------------- W3UWND
__global__ void uwnd_kernel(UwndArgs a) {
  WWB_GRID_LOOP(i, a.nsea) {
    if (a.flfrst) {  // :643-671, from WX0..DTN at (IX,IY) = MAPSF(ISEA,1:2)
      const int ix = a.mapsf[i] - 1, iy = a.mapsf[a.msea + i] - 1;
      const long long c = ix + static_cast<long long>(iy) * a.nx;
      const float wx0 = a.wx0[c], wy0 = a.wy0[c], wxn = a.wxn[c], wyn = a.wyn[c];
      const float ua0 = sqrtf(wx0 * wx0 + wy0 * wy0);
      const float uan = sqrtf(wxn * wxn + wyn * wyn);
      const float d0 = ua0 > 1.E-7f ? mod_tpi(kTpi + dm::atan2f(wy0, wx0)) : 0.0f;
      const float dn = uan > 1.E-7f ? mod_tpi(kTpi + dm::atan2f(wyn, wxn)) : d0;
      const float ud0 = ua0 > 1.E-7f ? d0 : dn;
      float dd = dn - ud0;
      if (fabsf(dd) > kPi) dd = dd - kTpi * copysignf(1.0f, dd);
      a.ua0[i] = ua0;
      a.uai[i] = uan - ua0;
      a.ud0[i] = ud0;
      a.udi[i] = dd;
      a.as0[i] = a.dt0[c];
      a.asi[i] = a.dtn[c] - a.dt0[c];
    }
    // :704-731, X = X0 + RD*XI
    const float ua = a.ua0[i] + a.rd * a.uai[i];
    const float ud = a.ud0[i] + a.rd * a.udi[i];
    a.ua[i] = ua;
    a.ud[i] = ud;
    a.as[i] = a.as0[i] + a.rd * a.asi[i];
    if (a.flcur) {  // :746-755, the wind relative to the current
      float sn, cs;
      dm::sincosf(ud, &sn, &cs);
      const float uxr = ua * cs - a.rwindc * a.cx[i];
      const float uyr = ua * sn - a.rwindc * a.cy[i];
      a.u10[i] = fmax2(0.001f, sqrtf(uxr * uxr + uyr * uyr));
      a.u10d[i] = mod_tpi(kTpi + dm::atan2f(uyr, uxr));
    } else {  // :766-769
      a.u10[i] = fmax2(0.001f, ua);
      a.u10d[i] = ud;
    }
  }
}

// ------------------------------------------------------------------------------------- W3DZXY
/// One output cell: tx, ty from the neighbours (a, b) and (c, d) of the cell, in the reference's
/// association: ((tx * DPDX) + (ty * DQDX)) * DFAC.
__device__ __forceinline__ void dzxy_out(const DzxyArgs& a, long long cell, float tx, float ty) {
  const float gx = (tx * a.dpdx[cell]) + (ty * a.dqdx[cell]);
  const float gy = (tx * a.dpdy[cell]) + (ty * a.dqdy[cell]);
  a.dzzdx[cell] = gx * a.dfac;
  a.dzzdy[cell] = gy * a.dfac;
}

/// :3364-3416 for IY = 2..NY-1, IX = ixstart..ixend.
__global__ void dzxy_kernel(DzxyArgs a, int ixstart, int ixend) {
  const int ny = a.ny, nx = a.nx;
  const long long nrow = ny - 2, ncol = ixend - ixstart + 1;
  WWB_GRID_LOOP(t, nrow * ncol) {
    const int iy = 2 + static_cast<int>(t % nrow), ix = ixstart + static_cast<int>(t / nrow);
    auto sta = [&](int jy, int jx) {
      return a.mapsta[(jy - 1) + static_cast<long long>(jx - 1) * ny];
    };
    auto zz = [&](int jy, int jx) {
      return a.zz[a.mapfs[(jy - 1) + static_cast<long long>(jx - 1) * ny] - 1];
    };
    if (sta(iy, ix) == 0) continue;
    float stx = 0.5f;
    const int ixps = (ix == nx) ? 1 : ix + 1;
    int ixp = ixps;
    if (sta(iy, ixps) == 0) {
      ixp = ix;
      stx = 1.0f;
    }
    const int ixms = (ix == 1) ? nx : ix - 1;
    int ixm = ixms;
    if (sta(iy, ixms) == 0) {
      ixm = ix;
      stx = 1.0f;
    }
    float sty = 0.5f;
    int iyp = iy + 1;
    if (sta(iy + 1, ix) == 0) {
      iyp = iy;
      sty = 1.0f;
    }
    int iym = iy - 1;
    if (sta(iy - 1, ix) == 0) {
      iym = iy;
      sty = 1.0f;
    }
    const float tx = (zz(iy, ixp) - zz(iy, ixm)) * stx;
    const float ty = (zz(iyp, ix) - zz(iym, ix)) * sty;
    dzxy_out(a, (iy - 1) + static_cast<long long>(ix - 1) * ny, tx, ty);
  }
}

/// :3422-3484, the tripole seam row IY = NY.
__global__ void dzxy_trpl_kernel(DzxyArgs a) {
  const int ny = a.ny, nx = a.nx, iy = ny;
  WWB_GRID_LOOP(t, nx) {
    const int ix = 1 + static_cast<int>(t);
    auto sta = [&](int jy, int jx) {
      return a.mapsta[(jy - 1) + static_cast<long long>(jx - 1) * ny];
    };
    auto zz = [&](int jy, int jx) {
      return a.zz[a.mapfs[(jy - 1) + static_cast<long long>(jx - 1) * ny] - 1];
    };
    if (sta(iy, ix) == 0) continue;
    float stx = 0.5f;
    const int ixps = (ix == nx) ? 1 : ix + 1;
    int ixp = ixps;
    if (sta(iy, ixps) == 0) {
      ixp = ix;
      stx = 1.0f;
    }
    const int ixms = (ix == 1) ? nx : ix - 1;
    int ixm = ixms;
    if (sta(iy, ixms) == 0) {
      ixm = ix;
      stx = 1.0f;
    }
    float sty = 0.5f;
    const int ixtrpls = nx - ix + 1;
    int ixtrpl = ixtrpls;
    if (sta(iy, ixtrpls) == 0) {
      ixtrpl = ix;
      sty = 1.0f;
    }
    int iym = iy - 1;
    if (sta(iy - 1, ix) == 0) {
      iym = iy;
      sty = 1.0f;
    }
    const float tx = (zz(iy, ixp) - zz(iy, ixm)) * stx;
    const float ty = (zz(iy, ixtrpl) - zz(iym, ix)) * sty;
    dzxy_out(a, (iy - 1) + static_cast<long long>(ix - 1) * ny, tx, ty);
  }
}

// ---------------------------------------------------------------------------- DISTAB
__global__ void distab_kernel(int nar1d, float dsie, float ecg0, float* ewn1, float* ecg1) {
  WWB_GRID_LOOP(t, nar1d + 1) {
    const int i = static_cast<int>(t);
    if (i == 0) {
      ewn1[0] = 0.0f;
      ecg1[0] = ecg0;
      continue;
    }
    const float si = static_cast<float>(i) * dsie;
    float k = 0.0f, cg = 0.0f;
    disp::wavnu2(si, 1.0f, k, cg, 1e-7f, 15);
    ewn1[i] = k;
    ecg1[i] = cg;
  }
}

/// max_r of the reference's W3CFLXY: a > b ? a : b (x86 MAXSS/MAXPS with a as destination), so a
/// NaN or a tie of zeros of opposite sign yields b, as the CPU code's operand order decides.
__device__ __forceinline__ float maxr(float a, float b) { return a > b ? a : b; }

/// The operands of one sea point's CFL numbers (prop_cflxy.hpp:28-48, w3pro3md.F90:2111-2127):
/// for a direction (ECOS, ESIN) and a group velocity CG(IK), the advection velocity
/// CXTOT = ECOS*CG/CLATS (- VGX/CLATS under W3_MGP, + CX/CLATS with currents), CYTOT likewise
/// without the latitude factor, and the two CFL numbers (CXTOT*DPDX + CYTOT*DPDY)*DTG and
/// (CXTOT*DQDX + CYTOT*DQDY)*DTG, every operation rounded on its own.
struct CflPoint {
  float clat, dpdx, dpdy, dqdx, dqdy, dtg, vgx, vgy, cxs, cys;
  bool flcur, mgp;
  __device__ __forceinline__ void at(float ec, float es, float cgk, float& vx, float& vy) const {
    float cxt = __fdiv_rn(__fmul_rn(ec, cgk), clat);
    float cyt = __fmul_rn(es, cgk);
    if (mgp) {
      cxt = __fsub_rn(cxt, __fdiv_rn(vgx, clat));
      cyt = __fsub_rn(cyt, vgy);
    }
    if (flcur) {
      cxt = __fadd_rn(cxt, __fdiv_rn(cxs, clat));
      cyt = __fadd_rn(cyt, cys);
    }
    vx = __fmul_rn(__fadd_rn(__fmul_rn(cxt, dpdx), __fmul_rn(cyt, dpdy)), dtg);
    vy = __fmul_rn(__fadd_rn(__fmul_rn(cxt, dqdx), __fmul_rn(cyt, dqdy)), dtg);
  }
};

/// W3CFLXY, one thread per sea point (ISEA = JSEA under W3_SHRD). CFLXYMAX starts at 0 and is
/// raised frequency by frequency in the order the reference's compiled loop takes
/// (prop_cflxy.hpp:61-135): for NTH >= 2 four running maxima per IK over the direction pairs
/// (lanes VLCFLX(ITH), VLCFLY(ITH), VLCFLX(ITH+1), VLCFLY(ITH+1)), each started from the value
/// after the previous IK and reduced as max(max(l3,l1), max(l2,l0)), then an odd last direction;
/// for NTH = 1 one scalar step. The order only shows for NaNs and signed zeros; it is kept so
/// that every output bit matches. ECOS/ESIN sit in shared memory (2*NTH floats).
__global__ void cflxy_kernel(CflxyArgs a) {
  extern __shared__ float trig[];
  const int nth = a.nth;
  for (int i = threadIdx.x; i < nth; i += blockDim.x) {
    trig[i] = a.ecos[i];
    trig[nth + i] = a.esin[i];
  }
  __syncthreads();
  const int isea = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (isea > a.nsea) return;
  const int ix = a.mapsf[isea - 1];
  const int iy = a.mapsf[static_cast<size_t>(a.msea) + isea - 1];
  const size_t ixy = static_cast<size_t>(ix - 1) * a.ny + (iy - 1);
  CflPoint q;
  q.clat = a.clats[isea];
  q.dpdx = a.dpdx[ixy];
  q.dpdy = a.dpdy[ixy];
  q.dqdx = a.dqdx[ixy];
  q.dqdy = a.dqdy[ixy];
  q.dtg = a.dtg;
  q.vgx = a.vgx;
  q.vgy = a.vgy;
  q.flcur = a.flcur;
  q.mgp = a.mgp;
  q.cxs = a.flcur ? a.cx[isea] : 0.0f;
  q.cys = a.flcur ? a.cy[isea] : 0.0f;
  const float* cg = a.cg + static_cast<size_t>(isea) * (a.nk + 2);
  const int npair = nth / 2;
  float c = 0.0f;
  for (int ik = 1; ik <= a.nk; ++ik) {
    const float cgk = cg[ik];
    float vx, vy;
    if (nth >= 2) {
      float m0 = c, m1 = c, m2 = c, m3 = c;
      for (int j = 0; j < npair; ++j) {
        float vx1, vy1;
        q.at(trig[2 * j], trig[nth + 2 * j], cgk, vx, vy);
        q.at(trig[2 * j + 1], trig[nth + 2 * j + 1], cgk, vx1, vy1);
        m0 = maxr(m0, vx);
        m1 = maxr(m1, vy);
        m2 = maxr(m2, vx1);
        m3 = maxr(m3, vy1);
      }
      c = maxr(maxr(m3, m1), maxr(m2, m0));
      if (nth & 1) {
        q.at(trig[nth - 1], trig[2 * nth - 1], cgk, vx, vy);
        c = maxr(c, a.flcur ? maxr(vx, vy) : maxr(vy, vx));
      }
    } else {
      q.at(trig[0], trig[1], cgk, vx, vy);
      c = maxr(c, (a.flcur || a.mgp) ? maxr(vx, vy) : maxr(vy, vx));
    }
  }
  a.cflxymax[isea - 1] = c;
}

}  // namespace

void launch_wave_gath(int nsea, int ny, size_t nf, const float* row, const int* ixy,
                      float* field, cudaStream_t s) {
  WWB_CHECK(cudaMemsetAsync(field, 0, nf * sizeof(float), s));
  if (nsea > 0) gath_kernel<<<blocks(nsea, 256), 256, 0, s>>>(nsea, ny, row, ixy, field);
  WWB_CHECK(cudaGetLastError());
}

void launch_wave_scat(int nsea, int ny, const int* mapsta, const float* field, const int* ixy,
                      float* row, cudaStream_t s) {
  if (nsea > 0) scat_kernel<<<blocks(nsea, 256), 256, 0, s>>>(nsea, ny, mapsta, field, ixy, row);
  WWB_CHECK(cudaGetLastError());
}

void launch_wave_uwnd(const UwndArgs& a, cudaStream_t s) {
  if (a.nsea > 0) uwnd_kernel<<<blocks(a.nsea, 256), 256, 0, s>>>(a);
  WWB_CHECK(cudaGetLastError());
}

void launch_wave_dzxy(const DzxyArgs& a, cudaStream_t s) {
  const size_t nc = static_cast<size_t>(a.nx) * a.ny;
  WWB_CHECK(cudaMemsetAsync(a.dzzdx, 0, nc * sizeof(float), s));
  WWB_CHECK(cudaMemsetAsync(a.dzzdy, 0, nc * sizeof(float), s));
  const int ixstart = (a.iclose == -1) ? 2 : 1;  // ICLO_NONE
  const int ixend = (a.iclose == -1) ? a.nx - 1 : a.nx;
  if (a.ny - 1 >= 2 && ixend >= ixstart) {
    const long long n = static_cast<long long>(a.ny - 2) * (ixend - ixstart + 1);
    dzxy_kernel<<<blocks(n, 256), 256, 0, s>>>(a, ixstart, ixend);
  }
  if (a.iclose == 8 && a.ny >= 2)  // ICLO_TRPL
    dzxy_trpl_kernel<<<blocks(a.nx, 256), 256, 0, s>>>(a);
  WWB_CHECK(cudaGetLastError());
}

void launch_wave_distab(int nar1d, float dsie, float ecg0, float* ewn1, float* ecg1,
                        cudaStream_t s) {
  distab_kernel<<<1, 128, 0, s>>>(nar1d, dsie, ecg0, ewn1, ecg1);
  WWB_CHECK(cudaGetLastError());
}

void launch_wave_cflxy(const CflxyArgs& a, cudaStream_t s) {
  if (a.nsea > 0)
    cflxy_kernel<<<blocks(a.nsea, 256), 256, 2 * a.nth * sizeof(float), s>>>(a);
  WWB_CHECK(cudaGetLastError());
}

}  // namespace wwb
