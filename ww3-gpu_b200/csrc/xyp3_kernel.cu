// ww3-gpu_b200/csrc/xyp3_kernel.cu
// W3XYP3 + W3QCK3 + W3GATH/W3SCAT for sm_100a, a chunk of spectral components at a time.
//
// The reference runs one component per team and the averaging of section 3.a (its "scatter":
// every sea point adds a share of its action to up to nine cells, w3pro3md.F90:1154-1276) on
// one thread in source order, because the shares that land on one cell must be added in that
// order to give the Fortran's bits (prop_xyp3.hpp:1154-1276 comments, and its closing note).
// Here every phase is data-parallel over (component, element):
//
//  * The averaging is turned around into an ordered gather: the thread of target cell T lists
//    the sea points that can reach it (T itself and its eight neighbours), orders them by their
//    position in MAPCXY (the loop order: central points, then near-coast points), and replays
//    each one's statements in source order (centre, then +1,+2,+3,+4,-1,-2,-3,-4 for a central
//    point; centre, then +1,-1,+2,-2,+3,-3,+4,-4 with the land redirection for a near-coast
//    one), adding only the shares that land on T, and restarting from AQ where a point under
//    MAPTRN assigns its centre. Every addition to T therefore happens with the same operands in
//    the same order as in the serial loop, so VQ(T) has the Fortran's bits.
//  * The boundary restore, the global closure of the averaging and the x GSQRT that follow
//    it are applied by the same thread to its own cell (the closure needs the ghost cell's
//    gathered value, which the thread gathers as well).
//  * W3QCK3's sweep is tiled in shared memory over the lon/lat grid: a CTA takes a tile of
//    32 rows x 8 columns of one component, stages Q and the CFL numbers of the tile and of its
//    halo (two cells up- and downstream along the sweep), computes the fluxes of the tile's
//    faces and of the one upstream halo face, and writes the propagated Q of its active cells
//    (and the unchanged Q of the others) into the component's second buffer; the buffers swap
//    after the sweep. The reference's flux loop reads only the Q from before the sweep and its
//    propagation loop writes each cell once, so reading one buffer and writing the other gives
//    its bits; the one face a tile cannot see (the closed grid's face west of column 1, which
//    is the face east of column NX) is computed from global memory. The faces and active cells
//    come from a dense map of MAPX2/MAPY2/MAPAXY (Xyp3Grid::cell_kind); the list kernels
//    (one thread per MAPX2/MAPY2/MAPAXY entry) remain for maps that name a cell twice.
//    The closure copies whole rows (a kernel over rows).
//  * The boundary update takes, for each boundary point, the value of the last IBI naming it
//    (the serial loop's last write), found on the host once per call.
// Arithmetic: the reference's per-element expressions and operand order (-fmad=false).
#include "xyp3_kernel.cuh"

#include <algorithm>
#include <climits>
#include <cmath>
#include <vector>

#include "wwb_common.hpp"

namespace wwb {

/// Constants of one component (W3XYP3 section 1.a, 1.c) and its buffers.
struct Comp {
  int isp, ik, ith, ntloc;
  float ecosi, esini, rntloc, dtloc, dtrad, fthx, fthy, fcgx, fcgy;
  float* q;  ///< the state (VQ)
  float* a;  ///< the other buffer (AQ after the averaging)
  float* vlcflx;
  float* vlcfly;
  float* fla;
  float* rdi;  ///< 4 x NSEA
  int* iixy;   ///< 4 x NSEA
  unsigned* tcode;  ///< NSEA: 8 x 4 bits, the neighbour index j of each averaging statement
};

namespace {

constexpr int kBlock = 256;
constexpr float kPi = static_cast<float>(3.141592653589793);
constexpr float kGrav = 9.806f;
constexpr float kTpiInv = 1.0f / (2.0f * kPi);
constexpr float kCg0Fac = 0.575f * kGrav;       // 0.575*GRAV as REAL
constexpr float kDera = kPi / 180.0f;           // DERA
constexpr float kRadius = 4.E7f * kTpiInv;      // RADIUS
constexpr float kDeraRadius = kDera * kRadius;  // DERA*RADIUS

__host__ __device__ __forceinline__ float max_r(float a, float b) { return a > b ? a : b; }
__host__ __device__ __forceinline__ float min_r(float a, float b) { return a < b ? a : b; }
__host__ __device__ __forceinline__ int fint(float x) {
  return (x > -2147483904.0f && x < 2147483648.0f) ? static_cast<int>(x) : INT_MIN;
}
__host__ __device__ __forceinline__ int nint_r(float x) {
  const float r = roundf(x);
  return (r > -9.2233715e18f && r < 9.2233715e18f)
             ? static_cast<int>(static_cast<long long>(r))
             : 0;
}
__device__ __forceinline__ float grid2(const float* x, int ny, int iy, int ix) {
  return x[(ix - 1) * ny + iy - 1];
}

int blocks_for(long long n) {
  const long long b = (n + kBlock - 1) / kBlock;
  return static_cast<int>(std::max(1LL, std::min(b, 1LL << 30)));
}

// ---- section 1.a: per-component constants ------------------------------------------------
__global__ void comp_setup_kernel(Xyp3Grid g, int ncomp, const int* __restrict__ isps,
                                  Comp* comps) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncomp) return;
  Comp& k = comps[c];
  const int isp = isps[c];
  k.isp = isp;
  k.ith = 1 + (isp - 1) % g.nth;
  k.ik = 1 + (isp - 1) / g.nth;
  const float cg0 = kCg0Fac / g.sig[1];
  const float cga = kCg0Fac / g.sig[k.ik];
  k.ecosi = g.ecos[k.ith - 1];
  k.esini = g.esin[k.ith - 1];
  const float cgx = k.ecosi * cga;
  const float cgy = k.esini * cga;
  float acgx, acgy, cxc, cyc;
  if (g.flcur != 0) {
    acgx = max_r(fabsf(cgx + g.cxmin), fabsf(cgx + g.cxmax));
    acgy = max_r(fabsf(cgy + g.cymin), fabsf(cgy + g.cymax));
    cxc = max_r(fabsf(g.cxmin), fabsf(g.cxmax));
    cyc = max_r(fabsf(g.cymin), fabsf(g.cymax));
  } else {
    acgx = fabsf(cgx);
    acgy = fabsf(cgy);
    cxc = 0.0f;
    cyc = 0.0f;
  }
  const float t1 = max_r(acgx, acgy);
  const float t2 = max_r(cxc, cyc);
  const float e = cg0 * 0.001f;
  const float t3 = max_r(e, t2);
  const float cgn = max_r(t1, t3);
  k.ntloc = 1 + fint(g.dtg / ((g.dtcfl * cg0) / cgn));
  k.rntloc = static_cast<float>(k.ntloc);
  k.dtloc = g.dtg / k.rntloc;
  k.dtrad = k.dtloc;
  if (g.flagll != 0) k.dtrad = k.dtloc / kDeraRadius;
  float fth = (g.wdth * g.dth) * k.dtloc;
  float fcg = ((g.wdcg * 0.5f) * (g.xfr - (1.0f / g.xfr))) * k.dtloc;
  if (g.flagll != 0) {
    fth = (fth / kRadius) / kDera;
    fcg = (fcg / kRadius) / kDera;
  }
  fcg = fcg / k.rntloc;
  k.fthx = -(k.esini * fth);
  k.fthy = k.ecosi * fth;
  k.fcgx = k.ecosi * fcg;
  k.fcgy = k.esini * fcg;
}

// ---- W3GATH, section 1.c stencil, section 2.a velocities, per (component, sea point) -----
__device__ __forceinline__ void corner(float dxcgc, float dycgc, int ny, int& iixa, int& iixb,
                                       float& rda, float& rdb) {
  const int ixc = (dxcgc < 0.0f) ? -ny : ny;
  const int iyc = (dycgc < 0.0f) ? -1 : 1;
  iixa = ixc + iyc;
  if (fabsf(dxcgc) > fabsf(dycgc)) {
    iixb = ixc;
    rda = fabsf(dycgc / dxcgc);
    rdb = fabsf(dxcgc);
  } else {
    iixb = iyc;
    rda = (fabsf(dycgc) > 1.E-5f) ? fabsf(dxcgc / dycgc) : 1.0f;
    rdb = fabsf(dycgc);
  }
}

// ---- the averaging's neighbourhood: T - D(j), j = 0..8 --------------------------------------
/// D(j) of the nine cells an averaging statement of a sea point can reach (the order in which
/// gather_cell lists candidate sources), as (DX, DY) with D = DX*NY + DY.
__device__ __constant__ const signed char kNbDx[9] = {0, 0, 0, 1, -1, 1, 1, -1, -1};
__device__ __constant__ const signed char kNbDy[9] = {0, 1, -1, 0, 0, 1, -1, 1, -1};

/// j with D(j) = off, for off one of the nine (NY >= 3 keeps them distinct).
__device__ __forceinline__ unsigned nb_index(int off, int ny) {
  if (off == 0) return 0;
  if (off == 1) return 1;
  if (off == -1) return 2;
  if (off == ny) return 3;
  if (off == -ny) return 4;
  if (off == ny + 1) return 5;
  if (off == ny - 1) return 6;
  if (off == -ny + 1) return 7;
  return 8;
}

/// MAPSTX(j), j in 1-2NY .. NY*(NX+2).
__device__ __forceinline__ int stx(const Xyp3Grid& g, int j) { return g.mapstx[j + 2 * g.ny - 1]; }

/// The cells the eight averaging statements of sea point S (cell IXY = S) send their shares to,
/// as nb_index codes in statement order (bits 4m..4m+3 for statement m): a central point
/// +I1 +I2 +I3 +I4 -I1 -I2 -I3 -I4 (:1166-1180), a near-coast one +I1 -I1 +I2 -I2 +I3 -I3 +I4
/// -I4 with a land target sent back to the centre (:1195-1270), as gather_cell replays them.
__device__ __forceinline__ unsigned statement_codes(const Xyp3Grid& g, int S, bool central, int i1,
                                                    int i2, int i3, int i4) {
  const int ny = g.ny;
  int t[8];
  if (central) {
    t[0] = i1; t[1] = i2; t[2] = i3; t[3] = i4;
    t[4] = -i1; t[5] = -i2; t[6] = -i3; t[7] = -i4;
  } else {
    auto diag = [&](int i, int sgn) {
      const int ixc = (ny ^ i) < 0 ? -ny : ny, iyc = i - ixc;
      return (stx(g, S + sgn * i) >= 1 &&
              !(stx(g, S + sgn * ixc) <= 0 && stx(g, S + sgn * iyc) <= 0))
                 ? sgn * i
                 : 0;
    };
    auto side = [&](int i, int sgn) { return stx(g, S + sgn * i) >= 1 ? sgn * i : 0; };
    t[0] = diag(i1, 1); t[1] = diag(i1, -1); t[2] = side(i2, 1); t[3] = side(i2, -1);
    t[4] = diag(i3, 1); t[5] = diag(i3, -1); t[6] = side(i4, 1); t[7] = side(i4, -1);
  }
  unsigned code = 0;
#pragma unroll
  for (int m = 0; m < 8; ++m) code |= nb_index(t[m], ny) << (4 * m);
  return code;
}

/// W3GATH's value of component isp (the l-th listed) at sea point isea: VA under W3_SHRD, this
/// rank's VA column or the received block of its owner under W3_MPI (prop3_shim.cpp:111-141).
__device__ __forceinline__ float va_get(const Xyp3Grid& g, const float* __restrict__ va, int isea,
                                        int l, int isp) {
  if (g.naproc == 0) return va[static_cast<size_t>(isea) * g.nspec + (isp - 1)];
  const int ip = (isea - 1) % g.naproc + 1, k = (isea - 1) / g.naproc + 1;
  if (ip == g.iaproc) return va[static_cast<size_t>(k) * g.nspec + (isp - 1)];
  return g.rbuf[static_cast<size_t>(g.poff[ip - 1]) + static_cast<size_t>(l) * g.nsealm + (k - 1)];
}

/// W3SCAT's store of v, the counterpart of va_get.
__device__ __forceinline__ void va_put(const Xyp3Grid& g, float* __restrict__ va, int isea, int l,
                                       int isp, float v) {
  if (g.naproc == 0) {
    va[static_cast<size_t>(isea) * g.nspec + (isp - 1)] = v;
    return;
  }
  const int ip = (isea - 1) % g.naproc + 1, k = (isea - 1) / g.naproc + 1;
  if (ip == g.iaproc)
    va[static_cast<size_t>(k) * g.nspec + (isp - 1)] = v;
  else
    g.sbuf[static_cast<size_t>(g.poff[ip - 1]) + static_cast<size_t>(l) * g.nsealm + (k - 1)] = v;
}

__global__ void sea_setup_kernel(Xyp3Grid g, int ncomp, int l0, Comp* comps,
                                 const float* __restrict__ va) {
  const long long n = static_cast<long long>(ncomp) * g.nsea;
  const int qoff = g.ny - 1;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < n;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int c = static_cast<int>(t / g.nsea);
    const int isea = 1 + static_cast<int>(t % g.nsea);
    const Comp& k = comps[c];
    const int ix = g.mapsf[isea - 1];
    const int iy = g.mapsf[g.nsea + isea - 1];
    const int ixy = g.mapsf[2 * g.nsea + isea - 1];
    const float clat = g.clats[isea];
    const float dpdx = grid2(g.dpdx, g.ny, iy, ix), dpdy = grid2(g.dpdy, g.ny, iy, ix);
    const float dqdx = grid2(g.dqdx, g.ny, iy, ix), dqdy = grid2(g.dqdy, g.ny, iy, ix);
    // Section 1.c, the averaging stencil (:983-1059).
    float tmpx = k.fthx / clat;
    float tmpy = k.fthy;
    const float dxcgn = dpdx * tmpx + dpdy * tmpy;
    const float dycgn = dqdx * tmpx + dqdy * tmpy;
    tmpx = k.fcgx / clat;
    tmpy = k.fcgy;
    const float dxcgs = dpdx * tmpx + dpdy * tmpy;
    const float dycgs = dqdx * tmpx + dqdy * tmpy;
    int i1, i2, i3, i4;
    float r1, r2, r3, r4;
    corner(dxcgn + dxcgs, dycgn + dycgs, g.ny, i1, i2, r1, r2);
    corner(dxcgn - dxcgs, dycgn - dycgs, g.ny, i3, i4, r3, r4);
    float* rd = k.rdi + (isea - 1);
    int* ii = k.iixy + (isea - 1);
    rd[0] = r1;
    rd[g.nsea] = r2;
    rd[2 * g.nsea] = r3;
    rd[3 * g.nsea] = r4;
    ii[0] = i1;
    ii[g.nsea] = i2;
    ii[2 * g.nsea] = i3;
    ii[3 * g.nsea] = i4;
    if (g.gather_order != nullptr)
      k.tcode[isea - 1] =
          statement_codes(g, ixy, g.sea_pos[isea - 1] <= g.ncent, i1, i2, i3, i4);
    // W3GATH then section 2.a (:1080-1137): this sea point's cell only.
    const float cgi = g.cg[isea * (g.nk + 2) + k.ik];
    const float v = va_get(g, va, isea, l0 + c, k.isp);
    k.q[ixy + qoff] = (v / cgi) * clat;
    float cxt = (k.ecosi * cgi) / clat;
    float cyt = k.esini * cgi;
    if (g.flcur != 0) {
      cxt = cxt + (g.cx[isea] / g.clats[isea]);
      cyt = cyt + g.cy[isea];
    }
    const float cp = cxt * dpdx + cyt * dpdy;
    const float cq = cxt * dqdx + cyt * dqdy;
    k.vlcflx[ixy - 1] = k.dtrad * cp;
    k.vlcfly[ixy - 1] = k.dtrad * cq;
  }
}

// ---- section 3.a: the averaging as an ordered gather ---------------------------------------
/// VQ(T) after the averaging loops of one component, from AQ = a (section 3.a.1, 3.a.2).
__device__ float gather_cell(const Xyp3Grid& g, const Comp& k, const float* __restrict__ a,
                             int T) {
  const int ny = g.ny, nxy = g.nx * g.ny, nsea = g.nsea, qoff = ny - 1;
  // The nine candidate sources T - d, ordered by their MAPCXY position (INT_MAX: none).
  int pos[9], src[9];
  const int d[9] = {0, 1, -1, ny, -ny, ny + 1, ny - 1, -ny + 1, -ny - 1};
#pragma unroll
  for (int j = 0; j < 9; ++j) {
    const int S = T - d[j];
    int p = INT_MAX;
    if (S >= 1 && S <= nxy) {
      const int isea = g.cell_sea[S - 1];
      if (isea > 0) {
        p = g.sea_pos[isea - 1];
        // A near-coast point with MAPSTA <= 0 is skipped by the loop (:1191).
        if (p > g.ncent && g.mapsta[S - 1] <= 0) p = INT_MAX;
      }
    }
    pos[j] = p;
    src[j] = S;
  }
  // Sorting network (9 inputs), constant indices only.
#define WWB_CX(i, j)                                   \
  if (pos[j] < pos[i]) {                               \
    const int tp = pos[i];                             \
    pos[i] = pos[j];                                   \
    pos[j] = tp;                                       \
    const int ts = src[i];                             \
    src[i] = src[j];                                   \
    src[j] = ts;                                       \
  }
  WWB_CX(0, 1) WWB_CX(3, 4) WWB_CX(6, 7) WWB_CX(1, 2) WWB_CX(4, 5) WWB_CX(7, 8)
  WWB_CX(0, 1) WWB_CX(3, 4) WWB_CX(6, 7) WWB_CX(0, 3) WWB_CX(3, 6) WWB_CX(0, 3)
  WWB_CX(1, 4) WWB_CX(4, 7) WWB_CX(1, 4) WWB_CX(2, 5) WWB_CX(5, 8) WWB_CX(2, 5)
  WWB_CX(1, 3) WWB_CX(5, 7) WWB_CX(2, 6) WWB_CX(4, 6) WWB_CX(2, 4) WWB_CX(2, 3)
  WWB_CX(5, 6)
#undef WWB_CX
  float acc = 0.0f;
#pragma unroll 1
  for (int j = 0; j < 9; ++j) {
    if (pos[j] == INT_MAX) break;
    const int S = src[j];
    const int isea = g.cell_sea[S - 1];
    if (g.maptrn[S - 1] != 0) {  // :1157-1158 and :1192-1193, an assignment of the centre
      if (S == T) acc = a[S + qoff];
      continue;
    }
    const float cgi = g.cg[isea * (g.nk + 2) + k.ik];
    const float* rd = k.rdi + (isea - 1);
    const int* ii = k.iixy + (isea - 1);
    const float rd1 = rd[0];
    const float rd2 = min_r(rd[nsea] * cgi, 1.0f);
    const float rd3 = rd[2 * nsea];
    const float rd4 = min_r(cgi * rd[3 * nsea], 1.0f);
    const float av = a[S + qoff];
    const int i1 = ii[0], i2 = ii[nsea], i3 = ii[2 * nsea], i4 = ii[3 * nsea];
    if (S == T) acc = acc + (((3.0f - rd2) - rd4) * av) / 3.0f;
    const float c1 = ((rd2 * av) * rd1) / 6.0f;
    const float c2 = (((1.0f - rd1) * av) * rd2) / 6.0f;
    const float c3 = ((rd4 * av) * rd3) / 6.0f;
    const float c4 = (((1.0f - rd3) * av) * rd4) / 6.0f;
    if (pos[j] <= g.ncent) {  // central point: +1 +2 +3 +4 -1 -2 -3 -4 (:1166-1180)
      if (S + i1 == T) acc = acc + c1;
      if (S + i2 == T) acc = acc + c2;
      if (S + i3 == T) acc = acc + c3;
      if (S + i4 == T) acc = acc + c4;
      if (S - i1 == T) acc = acc + c1;
      if (S - i2 == T) acc = acc + c2;
      if (S - i3 == T) acc = acc + c3;
      if (S - i4 == T) acc = acc + c4;
    } else {  // near coast: +1 -1 +2 -2 +3 -3 +4 -4, land targets back to the centre
      int ixc = (ny ^ i1) < 0 ? -ny : ny;
      int iyc = i1 - ixc;
      int t;
      t = (stx(g, S + i1) >= 1 && !(stx(g, S + ixc) <= 0 && stx(g, S + iyc) <= 0)) ? S + i1 : S;
      if (t == T) acc = acc + c1;
      t = (stx(g, S - i1) >= 1 && !(stx(g, S - ixc) <= 0 && stx(g, S - iyc) <= 0)) ? S - i1 : S;
      if (t == T) acc = acc + c1;
      t = (stx(g, S + i2) >= 1) ? S + i2 : S;
      if (t == T) acc = acc + c2;
      t = (stx(g, S - i2) >= 1) ? S - i2 : S;
      if (t == T) acc = acc + c2;
      ixc = (ny ^ i3) < 0 ? -ny : ny;
      iyc = i3 - ixc;
      t = (stx(g, S + i3) >= 1 && !(stx(g, S + ixc) <= 0 && stx(g, S + iyc) <= 0)) ? S + i3 : S;
      if (t == T) acc = acc + c3;
      t = (stx(g, S - i3) >= 1 && !(stx(g, S - ixc) <= 0 && stx(g, S - iyc) <= 0)) ? S - i3 : S;
      if (t == T) acc = acc + c3;
      t = (stx(g, S + i4) >= 1) ? S + i4 : S;
      if (t == T) acc = acc + c4;
      t = (stx(g, S - i4) >= 1) ? S - i4 : S;
      if (t == T) acc = acc + c4;
    }
  }
  return acc;
}

/// Sections 3.a-3.b up to the sweeps, per (component, cell T of VQ): the averaged value, the
/// boundary restore (:1280-1282), the global closure (:1286-1291) and x GSQRT (:1301-1306).
/// Reads the component's state k.q as AQ and writes the new state into k.a (swapped after).
__global__ void average_kernel(Xyp3Grid g, int ncomp, const Comp* comps, int itloc) {
  const int ny = g.ny, nx = g.nx, nxy = nx * ny;
  const int nq = ny * (nx + 3), qoff = ny - 1;
  const long long n = static_cast<long long>(ncomp) * nq;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < n;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int c = static_cast<int>(t / nq);
    const Comp& k = comps[c];
    if (itloc > k.ntloc) continue;
    const int T = static_cast<int>(t % nq) + 1 - ny;  // 1-NY .. NY*(NX+2)
    const float* a = k.q;
    float v = gather_cell(g, k, a, T);
    if (T >= 1 && T <= nxy) {
      if (g.mapsta[T - 1] == 2) v = a[T + qoff];
      if (g.global) {
        const int col = (T - 1) / ny + 1;
        if (col == 1) v = v + gather_cell(g, k, a, T + nxy);
        if (col == nx) v = v + gather_cell(g, k, a, T - nxy);
      }
      const int isea = g.cell_sea[T - 1];
      if (isea > 0) {
        const int ix = g.mapsf[isea - 1], iy = g.mapsf[g.nsea + isea - 1];
        v = v * grid2(g.gsqrt, ny, iy, ix);
      }
    }
    k.a[T + qoff] = v;
  }
}

/// The sources of every cell T in the averaging loop's order (Xyp3Grid::gather_order): the
/// candidates of gather_cell, sorted by MAPCXY position. Depends on the grid only.
__global__ void gather_order_kernel(Xyp3Grid g) {
  const int ny = g.ny, nxy = g.nx * g.ny;
  const long long nq = static_cast<long long>(ny) * (g.nx + 3);
  const long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (t >= nq) return;
  const int T = static_cast<int>(t) + 1 - ny;
  int pos[9], idx[9];
#pragma unroll
  for (int j = 0; j < 9; ++j) {
    const int S = T - (kNbDx[j] * ny + kNbDy[j]);
    int p = INT_MAX;
    if (S >= 1 && S <= nxy) {
      const int isea = g.cell_sea[S - 1];
      if (isea > 0) {
        p = g.sea_pos[isea - 1];
        if (p > g.ncent && g.mapsta[S - 1] <= 0) p = INT_MAX;  // skipped by the loop (:1191)
      }
    }
    pos[j] = p;
    idx[j] = j;
  }
  // Insertion sort by position (distinct for real sources).
  for (int a = 1; a < 9; ++a)
    for (int b = a; b > 0 && pos[b] < pos[b - 1]; --b) {
      const int tp = pos[b]; pos[b] = pos[b - 1]; pos[b - 1] = tp;
      const int ti = idx[b]; idx[b] = idx[b - 1]; idx[b - 1] = ti;
    }
  unsigned long long w = 0;
  for (int m = 0; m < 9; ++m)
    w |= static_cast<unsigned long long>(pos[m] == INT_MAX ? 0xFu : static_cast<unsigned>(idx[m]))
         << (4 * m);
  g.gather_order[t] = w;
}

/// Sections 3.a-3.b up to the sweeps as average_kernel, tiled in shared memory: a CTA takes
/// 32 rows x 8 columns of one component's FIELD (columns 0..NX+2); each sea point of the tile
/// and its one-cell halo computes its averaging shares once (the centre's and C1..C4, or its
/// MAPTRN value), then each cell of the tile adds the shares that reach it, source by source in
/// the loop's order (gather_order) and statement by statement (Comp::tcode), as gather_cell
/// does. The global closure's far-column terms go through gather_cell.
constexpr int kAvgY = 32, kAvgX = 8;
__global__ void __launch_bounds__(kAvgY * kAvgX)
    average_tile_kernel(Xyp3Grid g, const Comp* comps, int itloc, int nty) {
  constexpr int RY = kAvgY + 2, RX = kAvgX + 2;
  __shared__ float sh_c[5][RX][RY];  // the centre's share, C1..C4 (or AQ under MAPTRN)
  __shared__ unsigned sh_code[RX][RY];
  __shared__ unsigned char sh_flag[RX][RY];  // 1 MAPTRN, 2 central point
  const Comp& k = comps[blockIdx.y];
  if (itloc > k.ntloc) return;
  const int ny = g.ny, nx = g.nx, nxy = nx * ny, nsea = g.nsea, qoff = ny - 1;
  const int iy0 = 1 + (blockIdx.x % nty) * kAvgY, ix0 = (blockIdx.x / nty) * kAvgX;
  const float* __restrict__ a = k.q;
  for (int i = threadIdx.x; i < RX * RY; i += blockDim.x) {
    const int c = i / RY, r = i % RY;
    const long long S = static_cast<long long>(ix0 - 1 + c - 1) * ny + (iy0 - 1 + r);
    if (S < 1 || S > nxy) continue;  // never a source (gather_order lists real cells only)
    const int isea = g.cell_sea[S - 1];
    if (isea <= 0) continue;
    const float av = a[S + qoff];
    if (g.maptrn[S - 1] != 0) {
      sh_flag[c][r] = 1;
      sh_c[0][c][r] = av;
      continue;
    }
    const float cgi = g.cg[isea * (g.nk + 2) + k.ik];
    const float* rd = k.rdi + (isea - 1);
    const float rd1 = rd[0];
    const float rd2 = min_r(rd[nsea] * cgi, 1.0f);
    const float rd3 = rd[2 * nsea];
    const float rd4 = min_r(cgi * rd[3 * nsea], 1.0f);
    sh_c[0][c][r] = (((3.0f - rd2) - rd4) * av) / 3.0f;
    sh_c[1][c][r] = ((rd2 * av) * rd1) / 6.0f;
    sh_c[2][c][r] = (((1.0f - rd1) * av) * rd2) / 6.0f;
    sh_c[3][c][r] = ((rd4 * av) * rd3) / 6.0f;
    sh_c[4][c][r] = (((1.0f - rd3) * av) * rd4) / 6.0f;
    sh_code[c][r] = k.tcode[isea - 1];
    sh_flag[c][r] = g.sea_pos[isea - 1] <= g.ncent ? 2 : 0;
  }
  __syncthreads();
  const int r = threadIdx.x % kAvgY, cc = threadIdx.x / kAvgY;
  const int iy = iy0 + r, ix = ix0 + cc;
  if (iy > ny || ix > nx + 2) return;
  const int T = (ix - 1) * ny + iy;
  const unsigned long long word = g.gather_order[T + qoff];
  float acc = 0.0f;
#pragma unroll 1
  for (int m = 0; m < 9; ++m) {
    const unsigned j = static_cast<unsigned>(word >> (4 * m)) & 0xFu;
    if (j == 0xFu) break;
    const int sc = cc + 1 - kNbDx[j], sr = r + 1 - kNbDy[j];
    const unsigned f = sh_flag[sc][sr];
    if (f & 1u) {  // MAPTRN: the centre is assigned (:1157-1158, :1192-1193)
      if (j == 0) acc = sh_c[0][sc][sr];
      continue;
    }
    if (j == 0) acc = acc + sh_c[0][sc][sr];
    const unsigned code = sh_code[sc][sr];
#pragma unroll
    for (int st = 0; st < 8; ++st)
      if (((code >> (4 * st)) & 0xFu) == j)
        acc = acc + sh_c[1 + ((f & 2u) ? (st & 3) : (st >> 1))][sc][sr];
  }
  float v = acc;
  if (T >= 1 && T <= nxy) {
    if (g.mapsta[T - 1] == 2) v = a[T + qoff];
    if (g.global) {
      const int col = (T - 1) / ny + 1;
      if (col == 1) v = v + gather_cell(g, k, a, T + nxy);
      if (col == nx) v = v + gather_cell(g, k, a, T - nxy);
    }
    const int isea = g.cell_sea[T - 1];
    if (isea > 0) {
      const int sx = g.mapsf[isea - 1], sy = g.mapsf[g.nsea + isea - 1];
      v = v * grid2(g.gsqrt, ny, sy, sx);
    }
  }
  k.a[T + qoff] = v;
}

__global__ void comp_reset_kernel(int ncomp, Comp* comps, float* vq, float* aq, size_t nq) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncomp) return;
  comps[c].q = vq + c * nq;
  comps[c].a = aq + c * nq;
}

__global__ void swap_kernel(int ncomp, Comp* comps, int itloc) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncomp || itloc > comps[c].ntloc) return;
  float* t = comps[c].q;
  comps[c].q = comps[c].a;
  comps[c].a = t;
}

// ---- W3QCK3 (prop_qck3.hpp:60-224), per (component, element) ------------------------------
struct Sweep {
  int inc, close;
  const int* mapbou;
  int nb0, nb1, nb2;
  const float* trans;
  bool x;  ///< the x sweep (VLCFLX) or the y sweep (VLCFLY)
};

__global__ void qck3_zero_closure_kernel(Xyp3Grid g, int ncomp, const Comp* comps, int itloc,
                                         Sweep w) {
  const int ny = g.ny, nx = g.nx, my = ny;
  const int nfla = my * (nx + 1), qoff = my - 1;
  const long long n = static_cast<long long>(ncomp) * nfla;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < n;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int c = static_cast<int>(t / nfla);
    const Comp& k = comps[c];
    if (itloc > k.ntloc) continue;
    const int i = static_cast<int>(t % nfla);
    k.fla[i] = 0.0f;  // :1085
    if (w.close && i < ny) {  // :1087-1112, closure part 1, a row per thread
      const int iy = i + 1;
      float* q = k.q;
      float* cfll = w.x ? k.vlcflx : k.vlcfly;
      const int iad00 = -my, iad02 = my, iadn0 = iad00 + my * nx, iadn1 = my * nx,
                iadn2 = iad02 + my * nx;
      q[iy + iad00 + qoff] = q[iy + iadn0 + qoff];
      q[iy + iadn1 + qoff] = q[iy + qoff];
      q[iy + iadn2 + qoff] = q[iy + iad02 + qoff];
      cfll[iy + iadn1 - 1] = cfll[iy - 1];
    }
  }
}

__global__ void qck3_flux_kernel(Xyp3Grid g, int ncomp, const Comp* comps, int itloc, Sweep w) {
  const int qoff = g.ny - 1, foff = g.ny - 1, inc = w.inc;
  const long long n = static_cast<long long>(ncomp) * w.nb2;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < n;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int c = static_cast<int>(t / w.nb2);
    const Comp& k = comps[c];
    if (itloc > k.ntloc) continue;
    const int ip = 1 + static_cast<int>(t % w.nb2);
    const int ixy = w.mapbou[ip - 1];
    const float* q = k.q;
    const float* cfll = w.x ? k.vlcflx : k.vlcfly;
    if (ip <= w.nb0) {  // :1130-1172
      const float cfl = (cfll[ixy + inc - 1] + cfll[ixy - 1]) * 0.5f;
      const float s = copysignf(1.1f, cfl);
      const int ixyc = ixy - inc * fint(min_r(s, 0.0f));
      const float c2 = cfl * cfl;
      const float t1 = (1.0f - cfl) * q[ixy + inc + qoff];
      const float t2 = (cfl + 1.0f) * q[ixy + qoff];
      const float h1 = (t1 + t2) * 0.5f;
      const float h2 = (1.0f - c2) / 6.0f;
      const float qixyc = q[ixyc + qoff];
      const float d2 = (q[ixyc - inc + qoff] - qixyc * 2.0f) + q[ixyc + inc + qoff];
      const float qb = h1 - h2 * d2;
      const int ixyu = ixyc - inc * fint(s);
      const int ixyd = 2 * ixyc - ixyu;
      const float qixyu = q[ixyu + qoff];
      const float dq = q[ixyd + qoff] - qixyu;
      const float dqnz = copysignf(max_r(fabsf(dq), 1.E-15f), dq);
      const float qcn = min_r(max_r((qixyc - qixyu) / dqnz, -0.1f), 1.1f);
      const float qbn0 = max_r((qb - qixyu) / dqnz, qcn);
      const float u = min_r(qcn / max_r(fabsf(cfl), 1.E-10f), 1.0f);
      const float qbn = min_r(qbn0, u);
      const float qbr = qixyu + qbn * dq;
      const float cfac = static_cast<float>(fint(fabsf(qcn - 0.5f) * 2.0f));
      const float qb2 = qixyc * cfac + (1.0f - cfac) * qbr;
      k.fla[ixy + foff] = cfl * qb2;
    } else {  // :1187-1234, boundary above (CFL at IXY) or below (CFL at IXY+INC)
      const float cfl = ip <= w.nb1 ? cfll[ixy - 1] : cfll[ixy + inc - 1];
      const float s = copysignf(1.1f, cfl);
      const int ixyc = ixy - inc * fint(min_r(s, 0.0f));
      k.fla[ixy + foff] = q[ixyc + qoff] * cfl;
    }
  }
}

__global__ void qck3_prop_kernel(Xyp3Grid g, int ncomp, const Comp* comps, int itloc, Sweep w) {
  const int ny = g.ny, nxy = g.nx * g.ny, qoff = ny - 1, foff = ny - 1, inc = w.inc;
  const long long n = static_cast<long long>(ncomp) * g.nact;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < n;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int c = static_cast<int>(t / g.nact);
    const Comp& k = comps[c];
    if (itloc > k.ntloc) continue;
    const int ip = 1 + static_cast<int>(t % g.nact);
    const int ixy = g.mapaxy[ip - 1];
    // :1240-1247, closure part 2 (FLA column 0 <- column NX), read where it is used.
    int jm = ixy - inc;
    if (w.close && jm <= 0) jm += nxy;
    const float fm = k.fla[jm + foff];
    const float fp = k.fla[ixy + foff];
    const int jn = (fm > 0.0f) ? -1 : 0;
    const int jp = (fp < 0.0f) ? 1 : 0;
    const float tt = k.q[ixy + qoff] + fm * w.trans[static_cast<long>(jn + 1) * nxy + ixy - 1];
    const float u = tt - fp * w.trans[static_cast<long>(jp + 1) * nxy + ixy - 1];
    k.q[ixy + qoff] = max_r(u, 0.0f);
  }
}

// ---- x 1/GSQRT (:1368-1373) and the boundary update (:1395-1415), per sea point -----------
/// The value of sea point isea (cell ixy) after the sub-step's sweeps: the boundary input
/// interpolated in time where the point takes one (the last IBI naming it), else v / GSQRT.
__device__ __forceinline__ float finish_value(const Xyp3Grid& g, const Comp& k, int itloc,
                                              int isea, int ixy, float v) {
  const int ibi = g.flbpi ? g.bnd_last[isea - 1] : 0;
  if (ibi > 0) {
    float rd1 = g.dsec_bpi0 - ((g.dtg * static_cast<float>(k.ntloc - itloc)) / k.rntloc);
    float rd2 = g.dsec_bpin;
    if (rd2 > 0.001f) {
      const float qq = rd1 / rd2;
      rd2 = min_r(max_r(qq, 0.0f), 1.0f);
      rd1 = 1.0f - rd2;
    } else {
      rd1 = 0.0f;
      rd2 = 1.0f;
    }
    const float b0 = g.bbpi0[static_cast<size_t>(ibi) * g.nspec + k.isp - 1];
    const float bn = g.bbpin[static_cast<size_t>(ibi) * g.nspec + k.isp - 1];
    return (((b0 * rd1) + (bn * rd2)) / g.cg[isea * (g.nk + 2) + k.ik]) * g.clats[isea];
  }
  return v / g.gsqrt[ixy - 1];
}

// ---- W3QCK3 tiled in shared memory (the sweep's flux and propagation in one kernel) -------
constexpr int kTileY = 32, kTileX = 8;  // core tile: 32 rows (IY, the fast index) x 8 columns

/// The flux of one face of kind `kind` (Xyp3Grid::cell_kind) from the CFL numbers at the face's
/// cell and the next one along the sweep (cf0, cf1) and Q at offsets -1, 0, 1, 2 along it (q4):
/// prop_qck3.hpp:103-157 for interior faces (the UQ scheme), :162-186 for the boundary ones.
/// Every expression as in qck3_flux_kernel, with IXYC, IXYU, IXYD as offsets from the face.
__device__ __forceinline__ float qck3_face_flux(int kind, float cf0, float cf1, const float* q4) {
  if (kind == 0) return 0.0f;
  if (kind == 1) {
    const float cfl = (cf1 + cf0) * 0.5f;
    const float s = copysignf(1.1f, cfl);
    const int oc = -fint(min_r(s, 0.0f));  // IXYC = IXY + OC*INC
    const float c2 = cfl * cfl;
    const float t1 = (1.0f - cfl) * q4[2];
    const float t2 = (cfl + 1.0f) * q4[1];
    const float h1 = (t1 + t2) * 0.5f;
    const float h2 = (1.0f - c2) / 6.0f;
    const float qixyc = q4[oc + 1];
    const float d2 = (q4[oc] - qixyc * 2.0f) + q4[oc + 2];
    const float qb = h1 - h2 * d2;
    const int ou = oc - fint(s);
    const int od = 2 * oc - ou;
    const float qixyu = q4[ou + 1];
    const float dq = q4[od + 1] - qixyu;
    const float dqnz = copysignf(max_r(fabsf(dq), 1.E-15f), dq);
    const float qcn = min_r(max_r((qixyc - qixyu) / dqnz, -0.1f), 1.1f);
    const float qbn0 = max_r((qb - qixyu) / dqnz, qcn);
    const float u = min_r(qcn / max_r(fabsf(cfl), 1.E-10f), 1.0f);
    const float qbn = min_r(qbn0, u);
    const float qbr = qixyu + qbn * dq;
    const float cfac = static_cast<float>(fint(fabsf(qcn - 0.5f) * 2.0f));
    const float qb2 = qixyc * cfac + (1.0f - cfac) * qbr;
    return cfl * qb2;
  }
  const float cfl = kind == 2 ? cf0 : cf1;
  const float s = copysignf(1.1f, cfl);
  const int oc = -fint(min_r(s, 0.0f));
  return q4[oc + 1] * cfl;
}

/// The flux of face IXY (1..NX*NY) read from global memory: the closed grid's face east of
/// column NX, which the tile of column 1 needs as its face west of column 1.
__device__ __forceinline__ float qck3_face_global(const Xyp3Grid& g, const float* q,
                                                  const float* cfll, int ixy, int inc, int sh) {
  const int kind = (g.cell_kind[ixy - 1] >> sh) & 3;
  if (kind == 0) return 0.0f;
  const int qoff = g.ny - 1;
  const float q4[4] = {q[ixy - inc + qoff], q[ixy + qoff], q[ixy + inc + qoff],
                       q[ixy + 2 * inc + qoff]};
  return qck3_face_flux(kind, cfll[ixy - 1], cfll[ixy + inc - 1], q4);
}

/// One W3QCK3 sweep (X: along IX, INC = NY; else along IY, INC = 1) for one tile of one
/// component: blockIdx.y the component, blockIdx.x the tile (row blocks fastest). The tiles
/// cover Q's columns 0..NX+2 (the ghost columns are copied); k.q is read, k.a written.
template <bool X>
__global__ void __launch_bounds__(kTileY * kTileX)
    qck3_tile_kernel(Xyp3Grid g, const Comp* comps, int itloc, Sweep w, int nty, int fin) {
  constexpr int RY = kTileY + (X ? 0 : 4), RX = kTileX + (X ? 4 : 0);  // staged rows, columns
  constexpr int OY = X ? 0 : 2, OX = X ? 2 : 0;  // local position of the first core cell
  constexpr int SH = X ? 0 : 2;                  // the sweep's bits in cell_kind
  __shared__ float qs[RX][RY];
  __shared__ float cs[RX][RY];
  __shared__ float fs[RX][RY];  // the flux of the face at each local cell
  const Comp& k = comps[blockIdx.y];
  if (itloc > k.ntloc) return;
  const int ny = g.ny, nx = g.nx, nxy = nx * ny, qoff = ny - 1, inc = X ? ny : 1;
  const long long nq = static_cast<long long>(ny) * (nx + 3), n1 = static_cast<long long>(ny) * (nx + 1);
  const int iy0 = 1 + (blockIdx.x % nty) * kTileY;
  const int ix0 = (blockIdx.x / nty) * kTileX;
  const float* __restrict__ q = k.q;
  const float* __restrict__ cfll = X ? k.vlcflx : k.vlcfly;
  // Cell (r, c) of the staged block is IXY = (IX-1)*NY + IY with IY = IY0-OY+r, IX = IX0-OX+c,
  // the reference's linear index (a row outside 1..NY is a cell of the next or previous column,
  // as the linear offsets of the y sweep make it).
  for (int i = threadIdx.x; i < RX * RY; i += blockDim.x) {
    const int c = i / RY, r = i % RY;
    const long long ixy = static_cast<long long>(ix0 - OX + c - 1) * ny + (iy0 - OY + r);
    const long long qi = ixy + qoff;
    qs[c][r] = (qi >= 0 && qi < nq) ? q[qi] : 0.0f;
    cs[c][r] = (ixy >= 1 && ixy <= n1) ? cfll[ixy - 1] : 0.0f;
  }
  __syncthreads();
  // The faces at the core cells and at the one upstream halo cell along the sweep.
  constexpr int FR = X ? kTileY : kTileY + 1, FC = X ? kTileX + 1 : kTileX;
  for (int i = threadIdx.x; i < FR * FC; i += blockDim.x) {
    const int c = OX - (X ? 1 : 0) + i / FR, r = OY - (X ? 0 : 1) + i % FR;
    const long long f = static_cast<long long>(ix0 - OX + c - 1) * ny + (iy0 - OY + r);
    const int kind = (f >= 1 && f <= nxy) ? (g.cell_kind[f - 1] >> SH) & 3 : 0;
    float flux = 0.0f;
    if (kind != 0) {
      float q4[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) q4[j] = X ? qs[c - 1 + j][r] : qs[c][r - 1 + j];
      flux = qck3_face_flux(kind, cs[c][r], X ? cs[c + 1][r] : cs[c][r + 1], q4);
    }
    fs[c][r] = flux;
  }
  __syncthreads();
  // The core cells: W3QCK3's propagation loop (prop_qck3.hpp:190-214) at the active ones.
  const int r = threadIdx.x % kTileY, cc = threadIdx.x / kTileY;
  const int iy = iy0 + r, ix = ix0 + cc;
  if (iy > ny || ix > nx + 2) return;
  const int lr = OY + r, lc = OX + cc;
  const int ixy = (ix - 1) * ny + iy;
  float v = qs[lc][lr];
  if (ixy >= 1 && ixy <= nxy && (g.cell_kind[ixy - 1] & 16)) {
    const int jm = ixy - inc;
    const float fm = (w.close && jm <= 0) ? qck3_face_global(g, q, cfll, jm + nxy, inc, SH)
                                          : fs[lc - (X ? 1 : 0)][lr - (X ? 0 : 1)];
    const float fp = fs[lc][lr];
    const int jn = (fm > 0.0f) ? -1 : 0;
    const int jp = (fp < 0.0f) ? 1 : 0;
    const float tt = v + fm * w.trans[static_cast<long>(jn + 1) * nxy + ixy - 1];
    const float u = tt - fp * w.trans[static_cast<long>(jp + 1) * nxy + ixy - 1];
    v = max_r(u, 0.0f);
  }
  if (fin && ixy >= 1 && ixy <= nxy) {  // the sub-step's last sweep: finish_kernel's step here
    const int isea = g.cell_sea[ixy - 1];
    if (isea > 0) v = finish_value(g, k, itloc, isea, ixy, v);
  }
  k.a[ixy + qoff] = v;
}

/// The x sweep's closure part 1 (prop_qck3.hpp:87-112) alone, a row per thread: the tiled
/// sweep needs no zeroed FLA.
__global__ void qck3_closure_kernel(Xyp3Grid g, int ncomp, const Comp* comps, int itloc) {
  const int ny = g.ny, nx = g.nx, my = ny, qoff = my - 1;
  const long long n = static_cast<long long>(ncomp) * ny;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < n;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const Comp& k = comps[static_cast<int>(t / ny)];
    if (itloc > k.ntloc) continue;
    const int iy = static_cast<int>(t % ny) + 1;
    float* q = k.q;
    const int iad00 = -my, iad02 = my, iadn0 = iad00 + my * nx, iadn1 = my * nx,
              iadn2 = iad02 + my * nx;
    q[iy + iad00 + qoff] = q[iy + iadn0 + qoff];
    q[iy + iadn1 + qoff] = q[iy + qoff];
    q[iy + iadn2 + qoff] = q[iy + iad02 + qoff];
    k.vlcflx[iy + iadn1 - 1] = k.vlcflx[iy - 1];
  }
}

// ---- finish_value per sea point, when no tiled sweep took it -------------------------------
__global__ void finish_kernel(Xyp3Grid g, int ncomp, const Comp* comps, int itloc) {
  const long long n = static_cast<long long>(ncomp) * g.nsea;
  const int qoff = g.ny - 1;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < n;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int c = static_cast<int>(t / g.nsea);
    const Comp& k = comps[c];
    if (itloc > k.ntloc) continue;
    const int isea = 1 + static_cast<int>(t % g.nsea);
    const int ixy = g.mapsf[2 * g.nsea + isea - 1];
    k.q[ixy + qoff] = finish_value(g, k, itloc, isea, ixy, k.q[ixy + qoff]);
  }
}

// ---- section 4 and W3SCAT, per (component, sea point) --------------------------------------
__global__ void store_kernel(Xyp3Grid g, int ncomp, int l0, const Comp* comps,
                             float* __restrict__ va) {
  const long long n = static_cast<long long>(ncomp) * g.nsea;
  const int qoff = g.ny - 1;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < n;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int c = static_cast<int>(t / g.nsea);
    const Comp& k = comps[c];
    const int isea = 1 + static_cast<int>(t % g.nsea);
    const int ixy = g.mapsf[2 * g.nsea + isea - 1];
    const int st = g.mapsta[ixy - 1];
    float v = k.q[ixy + qoff];
    if (st > 0) {
      const float x = (g.cg[isea * (g.nk + 2) + k.ik] / g.clats[isea]) * v;
      v = max_r(x, 0.0f);
    }
    if (st != 0) va_put(g, va, isea, l0 + c, k.isp, v);
  }
}

// ---- MINVAL/MAXVAL of the currents -----------------------------------------------------------
__global__ void current_range_kernel(const float* __restrict__ cx, const float* __restrict__ cy,
                                     int nsea, float* out) {
  // out: cxmin, cxmax, cymin, cymax, counts of non-NaN x and y (as floats)
  __shared__ float sh[6][kBlock];
  float mn_x = INFINITY, mx_x = -INFINITY, mn_y = INFINITY, mx_y = -INFINITY, nx = 0, ny = 0;
  for (int i = threadIdx.x; i < nsea; i += blockDim.x) {
    const float a = cx[i + 1], b = cy[i + 1];
    if (a == a) {
      mn_x = a < mn_x ? a : mn_x;
      mx_x = a > mx_x ? a : mx_x;
      nx += 1.0f;
    }
    if (b == b) {
      mn_y = b < mn_y ? b : mn_y;
      mx_y = b > mx_y ? b : mx_y;
      ny += 1.0f;
    }
  }
  sh[0][threadIdx.x] = mn_x;
  sh[1][threadIdx.x] = mx_x;
  sh[2][threadIdx.x] = mn_y;
  sh[3][threadIdx.x] = mx_y;
  sh[4][threadIdx.x] = nx;
  sh[5][threadIdx.x] = ny;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 1; i < blockDim.x; ++i) {
      sh[0][0] = sh[0][i] < sh[0][0] ? sh[0][i] : sh[0][0];
      sh[1][0] = sh[1][i] > sh[1][0] ? sh[1][i] : sh[1][0];
      sh[2][0] = sh[2][i] < sh[2][0] ? sh[2][i] : sh[2][0];
      sh[3][0] = sh[3][i] > sh[3][0] ? sh[3][i] : sh[3][0];
      sh[4][0] += sh[4][i];
      sh[5][0] += sh[5][i];
    }
    for (int j = 0; j < 6; ++j) out[j] = sh[j][0];
  }
}

}  // namespace

size_t xyp3_bytes_per_component(const Xyp3Grid& g) {
  const size_t nq = static_cast<size_t>(g.ny) * (g.nx + 3);
  const size_t n1 = static_cast<size_t>(g.ny) * (g.nx + 1);
  return sizeof(float) * (2 * nq + 3 * n1 + 4 * static_cast<size_t>(g.nsea)) +
         sizeof(int) * 5 * static_cast<size_t>(g.nsea) + sizeof(Comp);
}

void launch_xyp3_gather_order(const Xyp3Grid& g, cudaStream_t s) {
  gather_order_kernel<<<blocks_for(static_cast<long long>(g.ny) * (g.nx + 3)), kBlock, 0, s>>>(g);
  WWB_CHECK(cudaGetLastError());
}

void xyp3_current_range(Xyp3Grid& g, cudaStream_t s) {
  float* d = nullptr;
  WWB_CHECK(cudaMalloc(&d, 6 * sizeof(float)));
  current_range_kernel<<<1, kBlock, 0, s>>>(g.cx, g.cy, g.nsea, d);
  float h[6];
  const cudaError_t e1 = cudaGetLastError();
  const cudaError_t e2 = cudaMemcpyAsync(h, d, sizeof h, cudaMemcpyDeviceToHost, s);
  const cudaError_t e3 = cudaStreamSynchronize(s);
  cudaFree(d);
  WWB_CHECK(e1);
  WWB_CHECK(e2);
  WWB_CHECK(e3);
  const float nan = std::nanf("");
  const float huge = 3.40282347e38f;
  g.cxmin = g.nsea <= 0 ? huge : (h[4] > 0 ? h[0] : nan);
  g.cxmax = g.nsea <= 0 ? -huge : (h[4] > 0 ? h[1] : nan);
  g.cymin = g.nsea <= 0 ? huge : (h[5] > 0 ? h[2] : nan);
  g.cymax = g.nsea <= 0 ? -huge : (h[5] > 0 ? h[3] : nan);
}

// ---- the components other ranks own, between the resident VA and a message buffer ----------
__global__ void va_components_kernel(bool unpack, float* __restrict__ va, int nspec, int nsealm,
                                     const int* __restrict__ isps, int nisp,
                                     float* __restrict__ buf) {
  const long long n = static_cast<long long>(nisp) * nsealm;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < n;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int j = static_cast<int>(t / nsealm);
    const int k = 1 + static_cast<int>(t % nsealm);
    float* v = va + static_cast<size_t>(k) * nspec + (isps[j] - 1);
    if (unpack)
      *v = buf[t];
    else
      buf[t] = *v;
  }
}

void launch_va_components(bool unpack, float* va, int nspec, int nsealm, const int* isps,
                          int nisp, float* buf, cudaStream_t s) {
  const long long n = static_cast<long long>(nisp) * nsealm;
  if (n <= 0) return;
  va_components_kernel<<<blocks_for(n), kBlock, 0, s>>>(unpack, va, nspec, nsealm, isps, nisp,
                                                        buf);
  WWB_CHECK(cudaGetLastError());
}

int setup_xyp3_chunk(const Xyp3Grid& g, Xyp3Chunk& ch, cudaStream_t s) {
  const int nc = ch.ncomp;
  if (nc <= 0) return 0;
  const size_t nq = static_cast<size_t>(g.ny) * (g.nx + 3);
  const size_t n1 = static_cast<size_t>(g.ny) * (g.nx + 1);
  // Per-component buffers and constants.
  std::vector<Comp> hc(nc);
  for (int c = 0; c < nc; ++c) {
    hc[c] = Comp{};
    hc[c].q = ch.vq + c * nq;
    hc[c].a = ch.aq + c * nq;
    hc[c].vlcflx = ch.vlcflx + c * n1;
    hc[c].vlcfly = ch.vlcfly + c * n1;
    hc[c].fla = ch.fla + c * n1;
    hc[c].rdi = ch.rdi + static_cast<size_t>(c) * 4 * g.nsea;
    hc[c].iixy = ch.iixy + static_cast<size_t>(c) * 4 * g.nsea;
    hc[c].tcode = ch.tcode + static_cast<size_t>(c) * g.nsea;
  }
  WWB_CHECK(cudaMemcpyAsync(ch.comp, hc.data(), sizeof(Comp) * nc, cudaMemcpyHostToDevice, s));
  comp_setup_kernel<<<(nc + 127) / 128, 128, 0, s>>>(g, nc, ch.isp, ch.comp);
  WWB_CHECK(cudaGetLastError());
  std::vector<Comp> back(nc);
  WWB_CHECK(cudaMemcpyAsync(back.data(), ch.comp, sizeof(Comp) * nc, cudaMemcpyDeviceToHost, s));
  WWB_CHECK(cudaStreamSynchronize(s));
  int ntmax = 0;
  for (const Comp& k : back) ntmax = std::max(ntmax, k.ntloc);
  return ntmax;
}

void launch_xyp3_chunk(const Xyp3Grid& g, const Xyp3Chunk& ch, float* va, int ntmax,
                       cudaStream_t s) {
  const int nc = ch.ncomp;
  if (nc <= 0) return;
  const size_t nq = static_cast<size_t>(g.ny) * (g.nx + 3);
  const size_t n1 = static_cast<size_t>(g.ny) * (g.nx + 1);
  // The sub-steps swap each component's two buffers: start from the set-up assignment.
  comp_reset_kernel<<<(nc + 127) / 128, 128, 0, s>>>(nc, ch.comp, ch.vq, ch.aq, nq);
  // FIELD = 0 (W3GATH), the four speed arrays = 0 (:944-947).
  WWB_CHECK(cudaMemsetAsync(ch.vq, 0, sizeof(float) * nq * nc, s));
  WWB_CHECK(cudaMemsetAsync(ch.vlcflx, 0, sizeof(float) * n1 * nc, s));
  WWB_CHECK(cudaMemsetAsync(ch.vlcfly, 0, sizeof(float) * n1 * nc, s));
  const long long nsea_c = static_cast<long long>(nc) * g.nsea;
  sea_setup_kernel<<<blocks_for(nsea_c), kBlock, 0, s>>>(g, nc, ch.l0, ch.comp, va);
  WWB_CHECK(cudaGetLastError());
  // YFIRST (:928-931): the same for every component; it alternates every sub-step.
  const int dttst = fint(g.dsec_day);
  bool yfirst = (nint_r(static_cast<float>(dttst) / g.dtg) % 2) == 0;
  const Sweep sx{g.ny, g.global, g.mapx2, g.nmx0, g.nmx1, g.nmx2, g.atrnx, true};
  const Sweep sy{1, 0, g.mapy2, g.nmy0, g.nmy1, g.nmy2, g.atrny, false};
  const long long nfla = static_cast<long long>(nc) * n1;
  for (int itloc = 1; itloc <= ntmax; ++itloc) {
    if (g.gather_order != nullptr) {
      const int nty = (g.ny + kAvgY - 1) / kAvgY, ntx = (g.nx + 3 + kAvgX - 1) / kAvgX;
      average_tile_kernel<<<dim3(static_cast<unsigned>(nty * ntx), static_cast<unsigned>(nc)),
                            kAvgY * kAvgX, 0, s>>>(g, ch.comp, itloc, nty);
    } else {
      average_kernel<<<blocks_for(static_cast<long long>(nc) * nq), kBlock, 0, s>>>(
          g, nc, ch.comp, itloc);
    }
    swap_kernel<<<(nc + 127) / 128, 128, 0, s>>>(nc, ch.comp, itloc);
    const Sweep order[2] = {yfirst ? sy : sx, yfirst ? sx : sy};
    auto runs = [&](const Sweep& w) { return w.x ? g.flcx != 0 : g.flcy != 0; };
    // The tiled path applies finish_value in the sub-step's last sweep.
    const int last = runs(order[1]) ? 1 : runs(order[0]) ? 0 : -1;
    const bool fused_finish = g.cell_kind != nullptr && last >= 0;
    for (int o = 0; o < 2; ++o) {
      const Sweep& w = order[o];
      if (!runs(w)) continue;
      if (g.cell_kind != nullptr) {
        if (w.close)
          qck3_closure_kernel<<<blocks_for(static_cast<long long>(nc) * g.ny), kBlock, 0, s>>>(
              g, nc, ch.comp, itloc);
        const int nty = (g.ny + kTileY - 1) / kTileY, ntx = (g.nx + 3 + kTileX - 1) / kTileX;
        const dim3 grid(static_cast<unsigned>(nty * ntx), static_cast<unsigned>(nc));
        const int fin = o == last ? 1 : 0;
        if (w.x)
          qck3_tile_kernel<true><<<grid, kTileY * kTileX, 0, s>>>(g, ch.comp, itloc, w, nty, fin);
        else
          qck3_tile_kernel<false><<<grid, kTileY * kTileX, 0, s>>>(g, ch.comp, itloc, w, nty, fin);
        swap_kernel<<<(nc + 127) / 128, 128, 0, s>>>(nc, ch.comp, itloc);
        continue;
      }
      qck3_zero_closure_kernel<<<blocks_for(nfla), kBlock, 0, s>>>(g, nc, ch.comp, itloc, w);
      if (w.nb2 > 0)
        qck3_flux_kernel<<<blocks_for(static_cast<long long>(nc) * w.nb2), kBlock, 0, s>>>(
            g, nc, ch.comp, itloc, w);
      if (g.nact > 0)
        qck3_prop_kernel<<<blocks_for(static_cast<long long>(nc) * g.nact), kBlock, 0, s>>>(
            g, nc, ch.comp, itloc, w);
    }
    if (!fused_finish)
      finish_kernel<<<blocks_for(nsea_c), kBlock, 0, s>>>(g, nc, ch.comp, itloc);
    WWB_CHECK(cudaGetLastError());
    yfirst = !yfirst;
  }
  store_kernel<<<blocks_for(nsea_c), kBlock, 0, s>>>(g, nc, ch.l0, ch.comp, va);
  WWB_CHECK(cudaGetLastError());
}

size_t xyp3_comp_bytes() { return sizeof(Comp); }

void run_xyp3_chunk(const Xyp3Grid& g, Xyp3Chunk& ch, float* va, cudaStream_t s) {
  const int ntmax = setup_xyp3_chunk(g, ch, s);
  launch_xyp3_chunk(g, ch, va, ntmax, s);
}

}  // namespace wwb
