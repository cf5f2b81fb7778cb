// ww3-gpu_b200/csrc/utrn_kernel.cu
// W3UTRN on sm_100a: the cell-boundary transparencies ATRNX/ATRNY of the PR3 propagation from
// the sub-grid obstructions TRNX/TRNY, the ice concentration (IC0) and icebergs.
//
// Reference: ww3-gpu kokkos/src/ww_kokkos/updt_utrn.hpp:61-362 (W3UTRN of w3updtmd.F90:2809-3194
// at WW3 03adda91). Every pass writes each output element at most once and reads only what an
// earlier pass finished, so one thread per cell or sea point in stream order reproduces the
// Fortran's bits; the expressions keep its operand order, the folded PARAMETERs their float
// bits, and expf is the glibc-equal device expf.
#include "utrn_kernel.cuh"

#include "libm_dev.cuh"
#include "wwb_common.hpp"

namespace wwb {
namespace {

// RADIUS and DERA as gfortran folds them (updt_utrn.hpp:48-54), the literals 1.E-6 and 0.0001.
constexpr float kRadius = 0x1.848fd6p+22f;
constexpr float kDera = 0x1.1df46ap-6f;
constexpr float kFiceTol = 0x1.0c6f7ap-20f;
constexpr float kBergScale = 0x1.a36e2ep-14f;

/// Fortran MIN/MAX of two REALs in the object's operand order: a NaN or a signed-zero tie
/// gives the first operand.
__device__ __forceinline__ float fmin2(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float fmax2(float a, float b) { return (b > a) ? b : a; }

/// IXN, IXP, IYN, IYP of a cell (1-based IXY = IY + (IX-1)*NY); IX == 1 is tested first.
struct Nb {
  int ixn, ixp, iyn, iyp;
};
__device__ __forceinline__ Nb neighbours(int ix, int iy, int ixy, int nx, int ny) {
  Nb n;
  if (ix == 1) {
    n.ixn = iy + (nx - 1) * ny;
    n.ixp = iy + ix * ny;
  } else if (ix == nx) {
    n.ixn = iy + (ix - 2) * ny;
    n.ixp = iy;
  } else {
    n.ixn = iy + (ix - 2) * ny;
    n.ixp = iy + ix * ny;
  }
  if (iy == 1) {
    n.iyn = ixy;
    n.iyp = ixy + 1;
  } else if (iy == ny) {
    n.iyn = ixy - 1;
    n.iyp = ixy;
  } else {
    n.iyn = ixy - 1;
    n.iyp = ixy + 1;
  }
  return n;
}

#define WWB_GRID_LOOP(i, lo, n)                                                       \
  for (int i = (lo) + static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x); i < (n); \
       i += static_cast<int>(gridDim.x * blockDim.x))

/// ATRNX = ATRNY = 1 in every cell and side (:2917-2918); TRIX = TRIY = 1 when ice is on.
__global__ void utrn_fill_kernel(int ncell, float* atrnx, float* atrny, float* trix, float* triy) {
  WWB_GRID_LOOP(i, 0, ncell) {
    for (int k = 0; k < 3; ++k) {
      atrnx[i + k * ncell] = 1.0f;
      atrny[i + k * ncell] = 1.0f;
    }
    if (trix) {
      trix[i] = 1.0f;
      triy[i] = 1.0f;
    }
  }
}

/// TRFLAG 1, 3, 5: transparencies at the cell boundaries (:2939-2962).
__global__ void utrn_bound_kernel(UtrnGrid g, const int* __restrict__ mapsf,
                                  const float* __restrict__ trnx, const float* __restrict__ trny,
                                  float* atrnx, float* atrny) {
  const int nc = g.nx * g.ny;
  WWB_GRID_LOOP(i, 0, g.nsea) {
    const int ix = mapsf[i], iy = mapsf[g.nsea + i], ixy = mapsf[2 * g.nsea + i];
    float xm, xp;
    if (ix == 1) {
      xm = trnx[iy + (g.nx - 1) * g.ny - 1];
      xp = trnx[ixy - 1];
    } else if (ix == g.nx) {
      xm = trnx[ixy - g.ny - 1];
      xp = trnx[iy - 1];
    } else {
      xm = trnx[ixy - g.ny - 1];
      xp = trnx[ixy - 1];
    }
    atrnx[(ixy - 1)] = xm;
    atrnx[(ixy - 1) + 2 * nc] = xp;
    // TRNY(IXY-1) is TRNY(0), the REAL before the array, for IXY = 1: the caller passes it.
    atrny[(ixy - 1)] = ixy >= 2 ? trny[ixy - 2] : g.trny_before;
    atrny[(ixy - 1) + 2 * nc] = trny[ixy - 1];
  }
}

/// Other TRFLAG values: transparencies at the cell centres (:2972-3035).
__global__ void utrn_center_kernel(UtrnGrid g, const int* __restrict__ mapsf,
                                   const int* __restrict__ mapsta, const float* __restrict__ trnx,
                                   const float* __restrict__ trny, float* atrnx, float* atrny) {
  const int nc = g.nx * g.ny, ny = g.ny, nx = g.nx;
  WWB_GRID_LOOP(i, 0, g.nsea) {
    const int ix = mapsf[i], iy = mapsf[g.nsea + i], ixy = mapsf[2 * g.nsea + i];
    const Nb n = neighbours(ix, iy, ixy, nx, ny);
    const float tx = 1.0f + trnx[ixy - 1];
    const float txn = trnx[n.ixn - 1];
    float xm = tx * txn / (1.0f + txn);
    const float txp = trnx[n.ixp - 1];
    float xp = tx * txp / (1.0f + txp);
    const float ty = 1.0f + trny[ixy - 1];
    const float tyn = trny[n.iyn - 1];
    float ym = ty * tyn / (1.0f + tyn);
    const float typ = trny[n.iyp - 1];
    float yp = ty * typ / (1.0f + typ);
    auto sta = [&](int jy, int jx) { return mapsta[(jx - 1) * ny + (jy - 1)]; };
    if (sta(iy, ix) == 2) {  // an active boundary point: inflow sides at an edge or land open
      if (ix == 1 || sta(iy, ix - 1) <= 0) xm = 1.0f;
      if (ix == nx || sta(iy, ix + 1) <= 0) xp = 1.0f;
      if (iy == 1 || sta(iy - 1, ix) <= 0) ym = 1.0f;
      if (iy == ny || sta(iy + 1, ix) <= 0) yp = 1.0f;
    }
    atrnx[(ixy - 1)] = xm;
    atrnx[(ixy - 1) + 2 * nc] = xp;
    atrny[(ixy - 1)] = ym;
    atrny[(ixy - 1) + 2 * nc] = yp;
  }
}

/// Ice and iceberg transparencies of each sea cell into TRIX/TRIY (:3066-3127).
__global__ void utrn_ice_kernel(UtrnGrid g, const int* __restrict__ mapsf,
                                const float* __restrict__ hpfac, const float* __restrict__ hqfac,
                                const float* __restrict__ ice, const float* __restrict__ berg,
                                float* trix, float* triy) {
  WWB_GRID_LOOP(i, 0, g.nsea) {
    const int ix = mapsf[i], iy = mapsf[g.nsea + i], ixy = mapsf[2 * g.nsea + i];
    const int c = (ix - 1) * g.ny + (iy - 1);
    float dx = hpfac[c], dy = hqfac[c];
    if (g.flagll) {
      dx = dx * kRadius * kDera;
      dy = dy * kRadius * kDera;
    }
    float tx = trix[ixy - 1], ty = triy[ixy - 1];
    const float ic = ice[i + 1];  // ICE(0:NSEA)
    if (ic > 0.0f) {
      if (g.ficel > 0.0f) {
        tx = dm::expf(-(ic * dx / g.ficel));
        ty = dm::expf(-(ic * dy / g.ficel));
      } else {  // Tolman (2003)
        float lice0 = g.fice0 * dx, licen = g.ficen * dx;
        tx = (licen - ic * dx) / (licen - lice0);
        lice0 = g.fice0 * dy;
        licen = g.ficen * dy;
        ty = (licen - ic * dy) / (licen - lice0);
      }
      tx = fmax2(0.0f, fmin2(1.0f, tx));
      ty = fmax2(0.0f, fmin2(1.0f, ty));
    }
    const float bg = berg[i];
    if (bg > 0.0f) {
      const float bf = bg * g.ffacberg;
      tx = tx * dm::expf(-(bf * dx * kBergScale));
      ty = ty * dm::expf(-(bf * dy * kBergScale));
    }
    trix[ixy - 1] = tx;
    triy[ixy - 1] = ty;
  }
}

/// The ice transparencies combined into ATRNX/ATRNY (:3140-3177), after every cell's TRIX.
__global__ void utrn_combine_kernel(UtrnGrid g, const int* __restrict__ mapsf,
                                    const float* __restrict__ trix,
                                    const float* __restrict__ triy, float* atrnx, float* atrny) {
  const int nc = g.nx * g.ny;
  WWB_GRID_LOOP(i, 0, g.nsea) {
    const int ix = mapsf[i], iy = mapsf[g.nsea + i], ixy = mapsf[2 * g.nsea + i];
    const Nb n = neighbours(ix, iy, ixy, g.nx, g.ny);
    const float tx = 1.0f + trix[ixy - 1];
    const float txn = trix[n.ixn - 1];
    atrnx[(ixy - 1)] = atrnx[(ixy - 1)] * tx * txn / (1.0f + txn);
    const float txp = trix[n.ixp - 1];
    atrnx[(ixy - 1) + 2 * nc] = atrnx[(ixy - 1) + 2 * nc] * tx * txp / (1.0f + txp);
    const float ty = 1.0f + triy[ixy - 1];
    const float tyn = triy[n.iyn - 1];
    atrny[(ixy - 1)] = atrny[(ixy - 1)] * ty * tyn / (1.0f + tyn);
    const float typ = triy[n.iyp - 1];
    atrny[(ixy - 1) + 2 * nc] = atrny[(ixy - 1) + 2 * nc] * ty * typ / (1.0f + typ);
  }
}

int blocks(long long n) {
  const long long b = (n + 255) / 256;
  return static_cast<int>(b < 1 ? 1 : (b > 8192 ? 8192 : b));
}

}  // namespace

bool utrn_needs_ice(const UtrnGrid& g) {
  return !(g.trflag < 3 || g.ficen - g.fice0 < kFiceTol);
}

void launch_utrn(const UtrnGrid& g, const int* mapsf, const int* mapsta, const float* trnx,
                 const float* trny, const float* hpfac, const float* hqfac, const float* ice,
                 const float* berg, float* atrnx, float* atrny, float* trix, float* triy,
                 cudaStream_t s) {
  const int ncell = g.nx * g.ny;
  const bool ice_on = g.trflag != 0 && utrn_needs_ice(g);
  utrn_fill_kernel<<<blocks(ncell), 256, 0, s>>>(ncell, atrnx, atrny, ice_on ? trix : nullptr,
                                                  ice_on ? triy : nullptr);
  WWB_CHECK(cudaGetLastError());
  if (g.trflag == 0) return;
  if (g.nsea > 0) {
    if (g.trflag == 1 || g.trflag == 3 || g.trflag == 5)
      utrn_bound_kernel<<<blocks(g.nsea), 256, 0, s>>>(g, mapsf, trnx, trny, atrnx, atrny);
    else
      utrn_center_kernel<<<blocks(g.nsea), 256, 0, s>>>(g, mapsf, mapsta, trnx, trny, atrnx,
                                                         atrny);
    WWB_CHECK(cudaGetLastError());
  }
  if (!ice_on || g.nsea <= 0) return;
  utrn_ice_kernel<<<blocks(g.nsea), 256, 0, s>>>(g, mapsf, hpfac, hqfac, ice, berg, trix, triy);
  utrn_combine_kernel<<<blocks(g.nsea), 256, 0, s>>>(g, mapsf, trix, triy, atrnx, atrny);
  WWB_CHECK(cudaGetLastError());
}

}  // namespace wwb
