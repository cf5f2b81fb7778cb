// ww3-gpu_b200/csrc/srce_point.cuh
// W3SRCE (the dynamic-substep source-term integration of one sea point: ST4 + the DIA + W3SLN1,
// W3SBT1, W3SDB1, MLIM, SEED) for one CTA, written once for the device and the host in the
// phase style of st4_point.cuh.
//
// Reference: ww3-gpu kokkos/src/ww_kokkos/srce_kernel.hpp:140-583 (SrcePoint: init, step_a,
// dia, step_c, finish; WW3 w3srcemd.F90:869-2350 at 03adda91), srce_db1.hpp:33-150,
// srce_bt1.hpp (W3SBT1), srce_ln1.hpp (W3SLN1), snl1_team.hpp:351-497 (the DIA, here in its
// row-shift form as in snl1_kernel.cu). Each statement keeps the reference's operand order;
// MAX/MIN sites keep its operand order (mx(a,b) = a > b ? a : b, mn(a,b) = a < b ? a : b).
//
// Layout of one point's working set (floats). What a serial chain reads, or what is read
// everywhere, sits in the CTA's shared memory; arrays that only parallel loops touch sit in the
// point's slice of a global scratch buffer, which stays in L2. That keeps the shared part near
// 37 KB at 36x36, so four CTAs share an SM.
//   shared      SPEC, LLWS (NSPEC ints), WN1 CG1 DAM CBETA WNF (NK), DIRF (NTH), the ST4 NK
//               work arrays, EB (NK doubles), and one region reused in turn by the four
//               ordered-sum term arrays, W3SPR4's chain terms, the DIA's UE, SA1 and SA2, and
//               the closing band sums
//   global      SPECINIT VSIN VDIN VSNL VDNL VSDB VSLN (NSPEC each), and one region reused in
//               turn by W3SIN4 (DSTAB), the DIA (DA1P DA1M DA2P DA2M, DA1C + DA2C, CON),
//               W3SDS4 (VSDS VDDS BRLAMBDA BTH PB PB2) and VSBT VDBT.
#pragma once

#include "snl1_kernel.cuh"
#include "st4_point.cuh"

namespace wwb {
namespace pt {

WWB_PD float mx(float a, float b) { return a > b ? a : b; }
WWB_PD float mn(float a, float b) { return a < b ? a : b; }

/// W3SRCE's own grid arrays (ww_srce_init), 0-based: sig[ik] = SIG(IK+1) etc.
struct SrceGrid {
  const float *sig, *dden, *ecos, *esin;
  const int* mapwn;
};

/// Per-point inputs and the step's flags.
struct SrceIn {
  int it, inflags24, flogrd57, flogrd58;
  float d_inp, u10abs, u10dir, as, ice, dtg, dair, coef;
};

/// The point's scalars, shared by the CTA. r holds W3SPR4's outputs under W3SRCE's names
/// (r.ustar = USTAR, r.usdir = USTDIR, r.wnmean = WNMEAN, ...).
struct SrceSh {
  Spr4Out r;
  float tauwx, tauwy, dtdyn, fcut, tauox, tauoy, tauwix, tauwiy, tauwnx, tauwny, phiaw, tws,
      phioc, phibbl, phice, tauocx, tauocy, fpi;
  int shave;
  float whitecap[4], taubbl[2], tauice[2];
  float depth, drat, icescaleln, icescalein, icescalenl, icescaleds;
  float fage, fhigh, dttot, dt, tauwax, tauway, hstot, vddb, afilt, dtred;
  int nsteps, nkh, nkh1, nspech, done, nscut;
  int sin4_valid;  ///< the last W3SIN4's outputs hold for the next step's first call
  float red[32];
  Sin4Sh sin4;
  Sds4Sh sds4;
};

/// An offset with this bit is into the point's global scratch, otherwise into its shared part.
constexpr int kInGlobal = 1 << 30;

/// Whether W3SRCE's working set is split between shared memory and global scratch (four CTAs
/// of 128 threads per SM) or held in shared memory whole (two CTAs of 256).
#ifndef WWB_SRCE_SPLIT
#define WWB_SRCE_SPLIT 1
#endif
constexpr bool kSrceSplit = WWB_SRCE_SPLIT != 0;

/// Offsets (in floats) of the working set; see the file header.
struct SrceLayout {
  int nspec, nk, nth;
  int spec, specinit, vsin, vdin, vsnl, vdnl, vsdb, vsln, llws;
  int wn1, cg1, dam, cbeta, wnf, dirf, sin4eb, spr4w, sds4w, sds4iw, ebd;
  int ser, ser_len;      ///< shared region of the serial chains' operands
  int trans, trans_len;  ///< global region of the parallel phases' arrays
  int total_s, total_g;  ///< floats of shared memory and of global scratch per point
};

/// Floats of the DIA's per-point scratch (row-shift form) in shared memory (UE, SA1, SA2: the
/// arrays its gathers read most) and in global memory (DA1P, DA1M, DA2P, DA2M, DA1C + DA2C,
/// CON).
WWB_PD int dia_shared(const Snl1Dev& p) {
  return (p.nfrhgh + 1) * p.nth + 2 * (p.nfrchg + 1) * p.nth;
}
WWB_PD int dia_global(const Snl1Dev& p) {
  return 4 * (p.nfrchg + 1) * p.nth + p.nspec + p.nk;
}

inline SrceLayout srce_layout(const st4::Params& q, const Snl1Dev& n, bool split = kSrceSplit) {
  SrceLayout L{};
  const int ns = q.nspec, nk = q.nk, nth = q.nth;
  auto r4 = [](int x) { return (x + 3) & ~3; };
  const int R = r4(ns);
  L.nspec = ns;
  L.nk = nk;
  L.nth = nth;
  int o = 0;  // shared
  L.spec = o; o += R;
  L.llws = o; o += R;
  L.wn1 = o; o += r4(nk);
  L.cg1 = o; o += r4(nk);
  L.dam = o; o += r4(nk);
  L.cbeta = o; o += r4(nk);
  L.wnf = o; o += r4(nk);
  L.dirf = o; o += r4(nth);
  L.sin4eb = o; o += r4(7 * nk);  // W3SIN4's NK work (sin4_nk_work)
  L.spr4w = o; o += r4(5 * nk + 4);
  L.sds4w = o; o += r4(18 * nk);
  L.sds4iw = o; o += r4(2 * nk);
  L.ebd = o; o += r4(2 * nk);  // NK doubles (8-byte aligned: o is a multiple of 4)
  L.ser = o;
  int sl = 4 * R;  // the ordered-sum terms; W3SPR4's two chain arrays; the band sums (3 NK)
  if (r4(dia_shared(n)) > sl) sl = r4(dia_shared(n));
  if (r4(3 * nk) > sl) sl = r4(3 * nk);
  L.ser_len = sl;
  o += sl;
  // The rest in global scratch, or (split false) after the shared part.
  const int flag = split ? kInGlobal : 0;
  int g = split ? 0 : o;
  L.specinit = flag | g; g += R;
  L.vsin = flag | g; g += R;
  L.vdin = flag | g; g += R;
  L.vsnl = flag | g; g += R;
  L.vdnl = flag | g; g += R;
  L.vsdb = flag | g; g += R;
  L.vsln = flag | g; g += R;
  L.trans = flag | g;
  int t = 6 * R;  // W3SDS4's outputs and NSPEC work; W3SIN4's DSTAB is 3 NSPEC
  if (r4(dia_global(n)) > t) t = r4(dia_global(n));
  L.trans_len = t;
  g += t;
  L.total_s = split ? o : g;
  L.total_g = split ? g : 0;
  return L;
}

// ---------------------------------------------------------------------------- the DIA, one point
/// W3SNL1 for one point in the row-shift form (the arithmetic of snl1_rowshift_kernel):
/// a (NSPEC), cg (NK) in; s, d (NSPEC) out; scratch dia_shared(p) floats in ss (UE, SA1, SA2)
/// and dia_global(p) floats in gs (DA1P, DA1M, DA2P, DA2M, DC = DA1C + DA2C, CON). DA1C and
/// DA2C are read back only at their own bin, so their sum is kept (the same two roundings).
WWB_PN void dia_point(const Cta& cta, const Snl1Dev& p, const float* a, const float* cg,
                      float kdmean, float* s, float* d, float* ss, float* gs) {
  const int nth = p.nth, nfr = p.nfr, nfrhgh = p.nfrhgh, nfrchg = p.nfrchg;
  const int nspec = p.nspec, nspecx = p.nspecx, nk = p.nk;
  const int alen = (nfrchg + 1) * nth;
  float* const ue = ss;
  float* const sa1 = ue + (nfrhgh + 1) * nth;
  float* const sa2 = sa1 + alen;
  float* const da1p = gs;
  float* const da1m = da1p + alen;
  float* const da2p = da1m + alen;
  float* const da2m = da2p + alen;
  float* const dc = da2m + alen;
  float* const conx = dc + nspec;
  PFOR(i, nth) {
    ue[i] = 0.0f;
    sa1[i] = sa2[i] = da1p[i] = da1m[i] = da2p[i] = da2m[i] = 0.0f;
  }
  PFOR(k, nk) conx[k] = kTpiInv / p.sig[k] * cg[k];
  // Section 1: CONS (snl1_team.hpp:383-390).
  const float x0 = p.kdcon * kdmean;
  const float xx = (x0 < p.kdmn) ? p.kdmn : x0;
  const float y0 = p.snls3 * xx;
  const float x2 = (-1.e15f < y0) ? y0 : -1.e15f;
  const float cons = p.snlc1 * (1.0f + p.snls1 / xx * (1.0f - p.snls2 * xx) * dm::expf(x2));
  cta.sync();
  PFOR(isp, nspec) ue[isp + nth] = a[isp] / conx[isp / nth];
  cta.sync();
  PFOR(col, nth) {
    float t = ue[nfr * nth + col];
    for (int r = nfr + 1; r <= nfrhgh; ++r) {
      t = t * p.fachfe;
      ue[r * nth + col] = t;
    }
  }
  cta.sync();
  const float dal1 = p.dal1, dal2 = p.dal2, dal3 = p.dal3;
  PFOR(isp, nspecx) {
    const int ifr0 = isp / nth, ith = isp - ifr0 * nth;
    int c[8];
    for (int n = 0; n < 8; ++n) {
      const int v = ith + p.shift[n];
      c[n] = v < 0 ? v + nth : (v >= nth ? v - nth : v);
    }
    const int r1 = p.ifrow[0 * nfrchg + ifr0] * nth;
    const int r2 = p.ifrow[1 * nfrchg + ifr0] * nth;
    const int r3 = p.ifrow[2 * nfrchg + ifr0] * nth;
    const int r4 = p.ifrow[3 * nfrchg + ifr0] * nth;
    const float e00 = ue[isp + nth];
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
    sa1[o] = factor * sa1b;
    sa2[o] = factor * sa2b;
    if (isp < nspec) dc[isp] = ca * (sa1a + sa1b) + ca * (sa2a + sa2b);
    da1p[o] = factor * (dal1 * e00 - dal3 * em1);
    da1m[o] = factor * (dal2 * e00 - dal3 * ep1);
    da2p[o] = factor * (dal1 * e00 - dal3 * em2);
    da2m[o] = factor * (dal2 * e00 - dal3 * ep2);
  }
  cta.sync();
  {
    PFOR(isp, nspec) {
      const int ifr0 = isp / nth, ith = isp - ifr0 * nth;
      int c[8];
      for (int n = 0; n < 8; ++n) {
        const int v = ith + p.shift[n];
        c[n] = v < 0 ? v + nth : (v >= nth ? v - nth : v);
      }
      const int r5 = p.ifrow[4 * nfrchg + ifr0] * nth;
      const int r6 = p.ifrow[5 * nfrchg + ifr0] * nth;
      const int r7 = p.ifrow[6 * nfrchg + ifr0] * nth;
      const int r8 = p.ifrow[7 * nfrchg + ifr0] * nth;
      const int o = isp + nth;
      s[isp] = conx[ifr0] * (-2.0f * (sa1[o] + sa2[o]) +
                             p.awg[0] * (sa1[r6 + c[5]] + sa2[r6 + c[1]]) +
                             p.awg[1] * (sa1[r6 + c[4]] + sa2[r6 + c[0]]) +
                             p.awg[2] * (sa1[r5 + c[5]] + sa2[r5 + c[1]]) +
                             p.awg[3] * (sa1[r5 + c[4]] + sa2[r5 + c[0]]) +
                             p.awg[4] * (sa1[r8 + c[3]] + sa2[r8 + c[7]]) +
                             p.awg[5] * (sa1[r8 + c[2]] + sa2[r8 + c[6]]) +
                             p.awg[6] * (sa1[r7 + c[3]] + sa2[r7 + c[7]]) +
                             p.awg[7] * (sa1[r7 + c[2]] + sa2[r7 + c[6]]));
      d[isp] = -2.0f * dc[isp] + p.swg[0] * (da1p[r6 + c[5]] + da2p[r6 + c[1]]) +
               p.swg[1] * (da1p[r6 + c[4]] + da2p[r6 + c[0]]) +
               p.swg[2] * (da1p[r5 + c[5]] + da2p[r5 + c[1]]) +
               p.swg[3] * (da1p[r5 + c[4]] + da2p[r5 + c[0]]) +
               p.swg[4] * (da1m[r8 + c[3]] + da2m[r8 + c[7]]) +
               p.swg[5] * (da1m[r8 + c[2]] + da2m[r8 + c[6]]) +
               p.swg[6] * (da1m[r7 + c[3]] + da2m[r7 + c[7]]) +
               p.swg[7] * (da1m[r7 + c[2]] + da2m[r7 + c[6]]);
    }
  }
  cta.sync();
}

// ------------------------------------------------------------------------------ W3SRCE, one point
/// Everything one point's integration reads: configuration, tables, inputs, working set.
struct SrceCtx {
  const srce::Params* p;
  const SrceGrid* g;
  const st4::Params* q;
  const Fields* f;
  const Snl1Dev* n;
  SrceIn in;
  float* w;   ///< the shared part of the working set (SrceLayout)
  float* gw;  ///< the global part
  const SrceLayout* L;
  SrceSh* sh;
};

WWB_PD float* at(const SrceCtx& x, int off) {
  return (off & kInGlobal) ? x.gw + (off & ~kInGlobal) : x.w + off;
}

/// W3SPR4 with W3SRCE's arguments (:1080, :1119, :1878, :2012).
WWB_PD void srce_spr4(const Cta& cta, const SrceCtx& x) {
  const SrceLayout& L = *x.L;
  // The ELCS / ELSN terms go to the shared serial region (free at every call site).
  spr4(cta, *x.q, *x.f, at(x, L.spec), at(x, L.cg1), at(x, L.wn1), x.in.u10abs, x.in.u10dir,
       x.sh->tauwx, x.sh->tauwy, reinterpret_cast<const int*>(at(x, L.llws)), x.sh->r,
       at(x, L.spr4w), at(x, L.ser));
}

/// W3SIN4 with W3SRCE's arguments (:1100, :1239, :2007).
WWB_PD void srce_sin4(const Cta& cta, const SrceCtx& x) {
  const SrceLayout& L = *x.L;
  SrceSh& s = *x.sh;
  sin4(cta, *x.q, *x.f, at(x, L.spec), at(x, L.cg1), at(x, L.wn1), 1, x.in.u10abs, s.r.ustar,
       s.drat, x.in.as, x.in.u10dir, s.r.z0, &s.tauwx, &s.tauwy, &s.tauwax, &s.tauway,
       at(x, L.vsin), at(x, L.vdin), reinterpret_cast<int*>(at(x, L.llws)), at(x, L.trans),
       at(x, L.sin4eb), s.sin4);
}

/// 1. Initialisation (:869-1179). spec holds the point's spectrum, wn1/cg1 its NK arrays; the
/// shared scalars hold the INOUT packet values.
WWB_PN void srce_init(const Cta& cta, const SrceCtx& x) {
  const srce::Params& p = *x.p;
  const SrceLayout& L = *x.L;
  SrceSh& s = *x.sh;
  const int nk = p.nk, nspec = p.nspec;
  float* const spec = at(x, L.spec);
  PFOR(is, nspec) {
    at(x, L.vsin)[is] = at(x, L.vdin)[is] = at(x, L.vsnl)[is] = at(x, L.vdnl)[is] = 0.0f;
    at(x, L.vsln)[is] = at(x, L.vsdb)[is] = 0.0f;
  }
  PFOR(ik, nk) {
    const float w = at(x, L.wn1)[ik];
    at(x, L.dam)[ik] = p.facp / (x.g->sig[ik] * (w * (w * w)));
  }
  if (cta.role(0)) {
    s.depth = mx(x.in.d_inp, p.dmin);
    s.drat = x.in.dair / kDwat;
    s.icescaleln = mx(mn(1.0f - x.in.ice * p.icescales[0], 1.0f), 0.0f);
    s.icescalein = mx(mn(1.0f - x.in.ice * p.icescales[1], 1.0f), 0.0f);
    s.icescalenl = mx(mn(1.0f - x.in.ice * p.icescales[2], 1.0f), 0.0f);
    s.icescaleds = mx(0.0f, mn(1.0f - x.in.ice * p.icescales[3], 1.0f));
    s.dtdyn = 0.0f;
    s.dttot = 0.0f;
    s.nsteps = 0;
    s.phiaw = 0.0f;
    s.r.charn = 0.0f;
    s.tws = 0.0f;
    s.phibbl = 0.0f;
    s.tauwix = s.tauwiy = s.tauwnx = s.tauwny = 0.0f;
    s.tauwax = s.tauway = 0.0f;
    s.taubbl[0] = s.taubbl[1] = s.tauice[0] = s.tauice[1] = 0.0f;
    s.phice = s.tauocx = s.tauocy = 0.0f;
    s.r.wnmean = 0.0f;
    s.r.dlwmean = 0.0f;
    s.vddb = 0.0f;
    for (int j = 0; j < 4; ++j) s.whitecap[j] = 0.0f;
    if (x.q->sintailpar[3] > 0.5f) {
      s.tauwx = 0.0f;
      s.tauwy = 0.0f;
    }
    if (x.in.it == 0) {
      s.tauwx = s.tauwy = 0.0f;
      s.r.ustar = 0.0f;
      s.r.usdir = 0.0f;
    }
  }
  {
    // LLWS is 1 at IT = 0 (:1073); otherwise the reference reads it unset at :1080, where only
    // FMEANWS depends on it and :1119 overwrites that: start from 0.
    int* const llws = reinterpret_cast<int*>(at(x, L.llws));
    PFOR(is, nspec) llws[is] = x.in.it == 0 ? 1 : 0;
  }
  cta.sync();
  if (x.in.it != 0) {
    srce_spr4(cta, x);
    if (x.q->sintailpar[3] > 0.5f) srce_sin4(cta, x);
  }
  srce_spr4(cta, x);
  PFOR(is, nspec) at(x, L.specinit)[is] = spec[is];
  if (cta.role(0)) {
    s.tws = 1.0f / s.r.fmeanws;
    s.fage = 0.0f;
    s.fhigh = mx((p.ffxfm + 0.0f) * mx(s.r.fmeanws, s.r.fmean1), p.ffxpm / s.r.ustar);
    s.done = 0;
    s.sin4_valid = 0;
  }
  cta.sync();
}

/// W3SLN1 (w3sln1md.F90:56-211) into VSLN.
WWB_PN void srce_ln1(const Cta& cta, const SrceCtx& x) {
  const srce::Params& p = *x.p;
  const SrceLayout& L = *x.L;
  SrceSh& s = *x.sh;
  const int nk = p.nk, nth = p.nth;
  auto fmin2 = [](float a, float b) { return (b < a) ? b : a; };
  auto fmax2 = [](float a, float b) { return (b > a) ? b : a; };
  float cosu, sinu;
  dm::sincosf(x.in.u10dir, &sinu, &cosu);
  float* const dirf = at(x, L.dirf);
  float* const wnf = at(x, L.wnf);
  PFOR(ith0, nth) {
    const float m = fmax2(0.0f, x.g->ecos[ith0] * cosu + x.g->esin[ith0] * sinu);
    const float m2 = m * m;
    dirf[ith0] = m2 * m2;
  }
  const float ustar = s.r.ustar;
  const float u2 = ustar * ustar;
  const float fac = p.slnc1 * (u2 * u2);
  const float ff1 = p.fspm * kGrav / (28.0f * ustar);
  const float ff2 = p.fshf * fmin2(x.g->sig[nk - 1], s.fhigh);
  const float ffilt = fmin2(2.0f * x.g->sig[nk - 1], fmax2(ff2, ff1));
  PFOR(ik0, nk) {
    const float rfr = x.g->sig[ik0] / ffilt;
    if (rfr < 0.5f) {
      wnf[ik0] = 0.0f;
    } else {
      const float r2 = rfr * rfr;
      const float rm4 = 1.0f / (r2 * r2);
      wnf[ik0] = fac / at(x, L.wn1)[ik0] * dm::expf(-rm4);
    }
  }
  cta.sync();
  PFOR(is, nk * nth) at(x, L.vsln)[is] = wnf[is / nth] * dirf[is - (is / nth) * nth];
  cta.sync();
}

/// 2. The start of a step (:1210-1239): the step count, W3SLN1, W3SIN4. W3SIN4 here reads
/// exactly what the previous step's closing W3SIN4 (:2007) read when no W3SPR4 ran after it
/// (:2012 runs only for SINTAILPAR(4) < 0.5): the spectrum, USTAR, Z0 and the wind are then
/// unchanged and its outputs (VSIN, VDIN, LLWS, TAUWX/Y, TAUWAX/Y) are still in place, so the
/// call is not repeated. The bits are the same either way.
WWB_PD void srce_step_a(const Cta& cta, const SrceCtx& x) {
  if (cta.role(0)) x.sh->nsteps = x.sh->nsteps + 1;
  if (x.p->ln1) srce_ln1(cta, x);
  if (!x.sh->sin4_valid) srce_sin4(cta, x);
}

/// The step's DIA (:1259-1263) with KDMEAN = WNMEAN * DEPTH.
WWB_PD void srce_dia(const Cta& cta, const SrceCtx& x) {
  const SrceLayout& L = *x.L;
  dia_point(cta, *x.n, at(x, L.spec), at(x, L.cg1), x.sh->r.wnmean * x.sh->depth,
            at(x, L.vsnl), at(x, L.vdnl), at(x, L.ser), at(x, L.trans));
}

/// The CTA-wide MIN of v over the threads' values with mn(), combined into *dst = mn(*dst, .).
WWB_PD void cta_min_into(const Cta& cta, float v, float* dst, float* red) {
#if defined(__CUDA_ARCH__)
  for (int o = 16; o > 0; o >>= 1) {
    const float u = __shfl_down_sync(0xffffffffu, v, o);
    v = mn(v, u);
  }
  if ((cta.tid & 31) == 0) red[cta.tid >> 5] = v;
  cta.sync();
  if (cta.tid == 0) {
    float m = *dst;
    for (int w = 0; w < (cta.nthr + 31) / 32; ++w) m = mn(m, red[w]);
    *dst = m;
  }
  cta.sync();
#else
  (void)red;
  (void)cta;
  *dst = mn(*dst, v);
#endif
}

/// 2b. After the DIA (:1303-1997): W3SDS4, W3SDB1, W3SBT1, the time step, the update, the
/// fluxes, W3SPR4, FHIGH, MLIM, SEED, the tail; then W3SIN4 (:2007) and the end test.
WWB_PN void srce_step_c(const Cta& cta, const SrceCtx& x) {
  const srce::Params& p = *x.p;
  const st4::Params& q = *x.q;
  const SrceLayout& L = *x.L;
  SrceSh& s = *x.sh;
  const int nk = p.nk, nth = p.nth, nspec = p.nspec;
  float* const spec = at(x, L.spec);
  float* const T = at(x, L.trans);
  const int R = (nspec + 3) & ~3;
  float* const vsds = T;
  float* const vdds = T + R;
  float* const brlambda = T + 2 * R;
  float* const vsbt = T + 3 * R;  // after W3SDS4 (its BTH, PB, PB2 live at 3R..5R)
  float* const vdbt = T + 4 * R;
  float* const S = at(x, L.ser);  // the ordered sums' terms, read by one thread each
  float* const t_phiaw = S;
  float* const t_phibbl = S + R;
  float* const t_wc = S + 2 * R;
  float* const t_hs = S + 3 * R;
  const float* const vsin = at(x, L.vsin);
  const float* const vdin = at(x, L.vdin);
  float* const vsnl = at(x, L.vsnl);
  float* const vdnl = at(x, L.vdnl);
  float* const vsln = at(x, L.vsln);
  float* const vsdb = at(x, L.vsdb);

  // W3SDS4 (:1303): its NK work in the persistent set, BTH, PB, PB2 at T + 3R.
  sds4(cta, q, *x.f, spec, at(x, L.wn1), at(x, L.cg1), s.r.ustar, s.r.usdir, s.depth,
       x.in.dair, s.r.dlwmean, x.in.flogrd57, x.in.flogrd58, vsds, vdds, brlambda, s.whitecap,
       at(x, L.sds4w), T + 3 * R, reinterpret_cast<int*>(at(x, L.sds4iw)), s.sds4);
  // W3SDB1 (:1321), W3SBT1 (:1339).
  {
    double* const eb = reinterpret_cast<double*>(at(x, L.ebd));
    const float emean = s.r.emean;
    const bool early = static_cast<double>(emean) < 0x1p-1022;
    if (!early) {
      PFOR(ik0, nk) {
        double e = 0.;
        for (int ith = 0; ith < nth; ++ith) e = e + static_cast<double>(spec[ith + ik0 * nth]);
        eb[ik0] = e;
      }
    }
    cta.sync();
    if (cta.role(0) && !early) {
      const double thr = static_cast<double>(0x1p-126f);
      double hm;
      if (p.fdonly != 0) {
        hm = static_cast<double>(p.sdbc2) * static_cast<double>(s.depth);
      } else {
        const float dpos = (s.depth > 0.0f) ? s.depth : 0.0f;
        const double wnm = static_cast<double>(s.r.wnmean);
        hm = static_cast<double>(p.sdbc2) / wnm * dm::tanh_d(wnm * static_cast<double>(dpos));
      }
      const double hrms = sqrt(8. * static_cast<double>(emean));
      double bb, b;
      if (hm > thr) {
        bb = hrms * hrms / (hm * hm);
        b = sqrt(bb);
      } else {
        bb = 0.;
        b = 0.;
      }
      double q0 = 0.;
      if (b <= 0.5) {
        q0 = 0.;
      } else if (b <= 1.) {
        const double t = 2. * b - 1.;
        q0 = t * t;
      }
      double qb;
      if (b <= 0.2) {
        qb = 0.;
      } else if (b < 1.) {
        const double arg = dm::exp_d((q0 - 1.) / bb);
        qb = q0 - bb * (q0 - arg) / (bb - arg);
        for (int is = 1; is <= 3; ++is) qb = dm::exp_d((qb - 1.) / bb);
      } else {
        qb = static_cast<double>(1.0f - 0x1p-126f);
      }
      double cbj = 0.;
      if (b != 1. && (bb > thr) && (fabs(bb - qb) > thr)) {
        if (bb < 1.0) {
          cbj = 2. * static_cast<double>(p.sdbc1) * qb * static_cast<double>(s.r.fmean) / bb;
        } else {
          cbj = 2. * static_cast<double>(p.sdbc1) * static_cast<double>(s.r.fmean) * bb;
        }
      }
      s.vddb = static_cast<float>(-cbj);
    }
    // W3SBT1's cut (serial search), in the same role.
    if (cta.role(1)) {
      const float depth = s.depth;
      const float* const wn = at(x, L.wn1);
      if (depth * wn[0] > 6.0f) {
        s.nscut = -1;
      } else {
        const float factor = p.sbtc1 / depth;
        int ik = 1;
        for (; ik <= nk; ++ik) {
          if (wn[ik - 1] * depth > 6.0f) break;
          const float xx = at(x, L.cg1)[ik - 1] * wn[ik - 1] / x.g->sig[ik - 1] - 0.5f;
          at(x, L.cbeta)[ik - 1] = factor * (xx > 0.0f ? xx : 0.0f);
        }
        s.nscut = (ik - 1) * nth;
      }
    }
    cta.sync();
    if (!early) {
      const float dval = s.vddb;
      PFOR(is, nspec) vsdb[is] = dval * spec[is];
    }
    const int nscut = s.nscut;
    PFOR(is, nspec) {
      float dv;
      if (nscut < 0) {
        dv = 0.0f;
      } else {
        dv = is < nscut ? at(x, L.cbeta)[x.g->mapwn[is] - 1] : 0.0f;
      }
      vdbt[is] = dv;
      vsbt[is] = nscut < 0 ? 0.0f : dv * spec[is];
    }
  }
  // The time-step limits (:1427-1437).
  if (cta.role(0)) {
    s.nkh = min_i(nk, fint(p.facti1 * dm::logf(mx(1.E-7f, s.fhigh)) + p.facti2));
    s.nkh1 = min_i(nk, s.nkh + 1);
    s.nspech = s.nkh1 * nth;
    s.dtred = mn(p.dtmax, x.in.dtg - s.dttot);
    s.afilt = mx(at(x, L.dam)[nk - 1], p.xflt * s.r.amax);
  }
  cta.sync();
  const int nspech = s.nspech;
  if (x.in.inflags24) {
    PFOR(is, nspech) {
      vsnl[is] = s.icescalenl * vsnl[is];
      vdnl[is] = s.icescalenl * vdnl[is];
      vsln[is] = s.icescaleln * vsln[is];
      at(x, L.vsin)[is] = s.icescalein * vsin[is];
      at(x, L.vdin)[is] = s.icescalein * vdin[is];
      vsds[is] = s.icescaleds * vsds[is];
      vdds[is] = s.icescaleds * vdds[is];
    }
    cta.sync();
  }
  // :1484-1533, the MIN over IS.
  {
    const float afilt = s.afilt;
    float loc = dm::asfloat(0x7f800000u);
    PFOR(is, nspech) {
      const float vs = (((vsln[is] + vsin[is]) + vsnl[is]) + vsds[is]) + vsbt[is];
      const float vd = ((vdin[is] + vdnl[is]) + vdds[is]) + vdbt[is];
      const float damax =
          mn(mx(p.xrel * at(x, L.specinit)[is], afilt), at(x, L.dam)[is / nth]);
      const float afac = 1.0f / mx(fabs_f(vs / damax), 1.E-10f);
      const float v = afac / mx(mn(vd, 0.0f) * afac + 1.0f, 1.E-10f);
      loc = mn(loc, v);
    }
    cta_min_into(cta, loc, &s.dtred, s.red);
  }
  if (cta.role(0)) {
    float dt = s.dtred;
    dt = mx(dt, 0.5f);
    s.dtdyn = s.dtdyn + dt;
    const float rest = x.in.dtg - s.dttot;
    const int idt = 1 + fint((rest * 0.99f) / dt);
    dt = rest / static_cast<float>(idt);
    const bool shave = dt < p.dtmin && dt < rest;
    s.shave = shave ? 1 : 0;
    dt = mx(mn(p.dtmin, rest), dt);
    s.dt = dt;
    s.dttot = s.dttot + dt;
  }
  cta.sync();
  // :1761-1808, the update.
  {
    const float dt = s.dt, hdt = dt;
    const bool shave = s.shave != 0;
    PFOR(is, nspech) {
      const float vs = (((vsln[is] + vsin[is]) + vsnl[is]) + vsds[is]) + vsbt[is];
      const float vd = ((vdin[is] + vdnl[is]) + vdds[is]) + vdbt[is];
      const float einc1 = (dt * vs) / mx(1.0f - hdt * vd, 1.0f);
      float v;
      if (shave) {
        const float einc2 = copysignf(mn(fabs_f(einc1), at(x, L.dam)[is / nth]), einc1);
        v = mx(spec[is] + einc2, 0.0f);
      } else {
        v = mx(spec[is] + einc1, 0.0f);
      }
      const float e2 = (dt * vsdb[is]) / mx(1.0f - hdt * s.vddb, 1.0f);
      spec[is] = mx(v + e2, 0.0f);
    }
    cta.sync();
    // :1815-1847: the ordered sums, their terms first.
    PFOR(is, nspec) {
      const int ik = is / nth;
      const float factor = x.g->dden[ik] / at(x, L.cg1)[ik];
      t_phiaw[is] = ((vsin[is] * dt) * factor) / mx(1.0f - vdin[is] * dt, 1.0f);
      t_phibbl[is] = ((vsbt[is] * dt) * factor) / mx(1.0f - vdbt[is] * dt, 1.0f);
      t_wc[is] = vsin[is] > 0.0f ? spec[is] * factor : -0.0f;
      t_hs[is] = spec[is] * factor;
    }
    cta.sync();
    if (cta.role(0)) {
      float v = s.phiaw;
WWB_UNROLL(8)
      for (int is = 0; is < nspec; ++is) v = t_phiaw[is] + v;
      s.phiaw = v;
    }
    if (cta.role(1)) {
      float v = s.phibbl;
WWB_UNROLL(8)
      for (int is = 0; is < nspec; ++is) v = v - t_phibbl[is];
      s.phibbl = v;
    }
    if (cta.role(2)) {
      float v = 0.0f;
WWB_UNROLL(8)
      for (int is = 0; is < nspec; ++is) v = v + t_wc[is];
      s.whitecap[2] = sqrt_f(v) * 4.0f;
    }
    if (cta.role(3)) {
      float v = 0.0f;
WWB_UNROLL(8)
      for (int is = 0; is < nspec; ++is) v = v + t_hs[is];
      s.hstot = sqrt_f(v) * 4.0f;
    }
    if (cta.role(4)) {
      s.tauwix = s.tauwix + (s.tauwx * s.drat) * dt;
      s.tauwiy = s.tauwiy + (s.tauwy * s.drat) * dt;
      s.tauwnx = s.tauwnx + (s.drat * s.tauwax) * dt;
      s.tauwny = s.tauwny + (s.drat * s.tauway) * dt;
    }
    cta.sync();
  }
  srce_spr4(cta, x);  // :1878
  if (cta.role(0)) {
    s.fage = p.ffxfa * dm::tanhf((((x.in.u10abs * 0.3f) * s.r.fmeanws) * kTpi) / kGrav);
    const float fh1 = (p.ffxfm + s.fage) * s.r.fmean1;
    const float fh2 = p.ffxpm / s.r.ustar;
    s.fhigh = mn(mx(fh1, fh2), x.g->sig[nk - 1]);
    s.nkh = max_i(min_i(s.nkh1, fint(p.facti1 * dm::logf(mx(1.E-7f, s.fhigh)) + p.facti2)), 2);
    s.afilt = 0.0f;  // reused below as the MLIM flag / EM
    s.dtred = -1.0f;
    if (s.dttot >= x.in.dtg * 0.9999f) {
      const float hm = (p.fhmax * dm::tanhf(mx(0.0f, x.in.d_inp) * s.r.wnmean)) /
                       mx(s.r.wnmean, 9.99999974737875163555145263671875e-5f);
      const float em = (hm * hm) * 6.25e-2f;
      if (s.r.emean > em && s.r.emean > 1.E-30f) {
        s.dtred = em;  // MLIM applies with EM
      }
    }
  }
  cta.sync();
  if (s.dtred >= 0.0f) {
    const float em = s.dtred, emean = s.r.emean;
    PFOR(is, nspec) spec[is] = em * (spec[is] / emean);
    cta.sync();
    if (cta.role(0)) s.r.emean = em;
    cta.sync();
  }
  if (p.seed) {
    const int ik_lo = min_i(nk, s.nkh);
    PFOR(e, (nk - ik_lo + 1) * nth) {
      const int ik = ik_lo + e / nth, ith = e - (e / nth) * nth + 1;
      const float uc = (p.facsd * kGrav) / x.g->sig[ik - 1];
      const float w = at(x, L.wn1)[ik - 1];
      float slev = ((mn(mx(x.in.u10abs / uc - 1.0f, 0.0f), 1.0f) * 6.25E-4F) / ((w * w) * w)) /
                   x.g->sig[ik - 1];
      if (x.in.inflags24) slev = (1.0f - x.in.ice) * slev;
      float sn, cs;
      dm::sincosf(x.in.u10dir - x.f->th[ith - 1], &sn, &cs);
      const float c = mx(cs, 0.0f);
      const int is = ith + (ik - 1) * nth - 1;
      spec[is] = mx(slev * (c * c), spec[is]);
    }
    cta.sync();
  }
  // :1985-1997, the tail: a recurrence up the frequencies, parallel over directions.
  {
    const int nkh = s.nkh;
    PFOR(ith, nth) {
      for (int ik = nkh; ik < nk; ++ik)
        spec[ith + ik * nth] = spec[ith + (ik - 1) * nth] * p.fachfa + 0.0f;
    }
    cta.sync();
  }
  srce_sin4(cta, x);  // :2007
  if (q.sintailpar[3] < 0.5f) srce_spr4(cta, x);  // :2012
  if (cta.role(0)) {
    s.done = s.dttot >= 0.9999f * x.in.dtg ? 1 : 0;
    s.sin4_valid = q.sintailpar[3] < 0.5f ? 0 : 1;
  }
  cta.sync();
}

/// 3. After the loop (:2050-2350), FLD2 excepted (ww_srce_init refuses it).
WWB_PN void srce_finish(const Cta& cta, const SrceCtx& x) {
  const srce::Params& p = *x.p;
  const SrceLayout& L = *x.L;
  SrceSh& s = *x.sh;
  const int nk = p.nk, nth = p.nth, nspec = p.nspec;
  float* const spec = at(x, L.spec);
  const float* const specinit = at(x, L.specinit);
  float* const T = at(x, L.ser);  // per-IK band sums: eband, a1band, b1band
  PFOR(ik, nk) {
    float eband = 0.0f, a1band = 0.0f, b1band = 0.0f;
    for (int ith = 0; ith < nth; ++ith) {
      const float diff = specinit[ith + ik * nth] - spec[ith + ik * nth];
      eband = diff + eband;
      a1band = x.g->ecos[ith] * diff + a1band;
      b1band = x.g->esin[ith] * diff + b1band;
    }
    T[3 * ik] = eband;
    T[3 * ik + 1] = a1band;
    T[3 * ik + 2] = b1band;
  }
  cta.sync();
  if (cta.role(0)) {
    s.dtdyn = s.dtdyn / static_cast<float>(max_i(s.nsteps, 1));
    s.fcut = s.fhigh * kTpiInv;
    float efinish = 0.0f, mwxfinish = 0.0f, mwyfinish = 0.0f;
    for (int ik = 0; ik < nk; ++ik) {
      const float dden = x.g->dden[ik], cg = at(x, L.cg1)[ik], wn = at(x, L.wn1)[ik];
      efinish = (dden * T[3 * ik]) / cg + efinish;
      mwxfinish = (((dden * T[3 * ik + 1]) / cg) * wn) / x.g->sig[ik] + mwxfinish;
      mwyfinish = (wn * ((dden * T[3 * ik + 2]) / cg)) / x.g->sig[ik] + mwyfinish;
    }
    const float dtg = x.in.dtg;
    s.tauox = ((s.tauwix + mwxfinish * kGrav) - s.taubbl[0]) / dtg;
    s.tauoy = ((s.tauwiy + mwyfinish * kGrav) - s.taubbl[1]) / dtg;
    s.tauwix = s.tauwix / dtg;
    s.tauwiy = s.tauwiy / dtg;
    s.tauwnx = s.tauwnx / dtg;
    s.tauwny = s.tauwny / dtg;
    s.taubbl[0] = s.taubbl[0] / dtg;
    s.taubbl[1] = s.taubbl[1] / dtg;
    float c, sn;
    dm::sincosf(s.r.usdir, &sn, &c);
    const float k = s.r.ustar * (s.r.ustar * (x.in.coef * (x.in.dair * x.in.coef)));
    s.tauocx = k * c + (s.tauox - s.tauwix) * kDwat;
    s.tauocy = k * sn + (s.tauoy - s.tauwiy) * kDwat;
    const float dg = kDwat * kGrav;
    s.phioc = (((s.phiaw + efinish) - s.phibbl) * dg) / dtg;
    s.phiaw = (s.phiaw * dg) / dtg;
    s.phibbl = (s.phibbl * dg) / dtg;
    // The ice block without dispersion (:2124-2259): ATT = 1, SPEC unchanged; the sums are of
    // zeros and kept for their signed zeros.
    if (x.in.inflags24 && x.in.ice > 0.0f && !p.ic_numerics) {
      s.tauice[0] = s.tauice[1] = 0.0f;
      s.phice = 0.0f;
      for (int ik = 0; ik < nk; ++ik) {
        const float factor = x.g->dden[ik] / at(x, L.cg1)[ik];
        const float factor2 = ((factor * kGrav) * at(x, L.wn1)[ik]) / x.g->sig[ik];
        for (int ith = 0; ith < nth; ++ith) {
          const int is = ith + ik * nth;
          const float sp2 = spec[is];
          const float spn = static_cast<float>(1.0 * static_cast<double>(sp2));
          s.phice = s.phice + (spn - sp2) * factor;
          s.tauice[0] = s.tauice[0] - ((spn - sp2) * factor2) * x.g->ecos[is];
          s.tauice[1] = s.tauice[1] - ((spn - sp2) * factor2) * x.g->esin[is];
        }
      }
      s.phice = (((-1.0f * kDwat) * kGrav) * s.phice) / dtg;
      s.tauice[0] = s.tauice[0] / dtg;
      s.tauice[1] = s.tauice[1] / dtg;
    }
  }
  cta.sync();
  if (x.in.it == 0) {
    PFOR(is, nspec) spec[is] = specinit[is];
    cta.sync();
  }
  const int nlast = (nspec % 4 == 3) ? nspec - 1 : nspec;
  PFOR(is, nspec) spec[is] = is < nlast ? mx(spec[is], 0.0f) : mx(0.0f, spec[is]);
  cta.sync();
}

/// The step's flags and a point's PIN packet (ww_kokkos_c.hpp:231-240).
WWB_PD SrceIn srce_in(int it, int inflags24, int flogrd57, int flogrd58, float dtg,
                      const float* pin) {
  SrceIn in{};
  in.it = it;
  in.inflags24 = inflags24;
  in.flogrd57 = flogrd57;
  in.flogrd58 = flogrd58;
  in.dtg = dtg;
  in.d_inp = pin[srce::IN_D_INP];
  in.u10abs = pin[srce::IN_U10ABS];
  in.u10dir = pin[srce::IN_U10DIR];
  in.as = pin[srce::IN_AS];
  in.ice = pin[srce::IN_ICE];
  in.dair = pin[srce::IN_DAIR];
  in.coef = pin[srce::IN_COEF];
  return in;
}

/// A point's INOUT scalars (PSC packet, WHITECAP, TAUBBL, TAUICE) into the shared state, and
/// back with SHAVE (single thread).
WWB_PD void srce_psc_in(SrceSh& s, const float* psc, const float* wc, const float* tb,
                        const float* ti) {
  s.r.ustar = psc[srce::SC_USTAR];
  s.r.usdir = psc[srce::SC_USTDIR];
  s.tauwx = psc[srce::SC_TAUWX];
  s.tauwy = psc[srce::SC_TAUWY];
  s.dtdyn = psc[srce::SC_DTDYN];
  s.fcut = psc[srce::SC_FCUT];
  s.tauox = psc[srce::SC_TAUOX];
  s.tauoy = psc[srce::SC_TAUOY];
  s.tauwix = psc[srce::SC_TAUWIX];
  s.tauwiy = psc[srce::SC_TAUWIY];
  s.tauwnx = psc[srce::SC_TAUWNX];
  s.tauwny = psc[srce::SC_TAUWNY];
  s.phiaw = psc[srce::SC_PHIAW];
  s.r.charn = psc[srce::SC_CHARN];
  s.tws = psc[srce::SC_TWS];
  s.phioc = psc[srce::SC_PHIOC];
  s.phibbl = psc[srce::SC_PHIBBL];
  s.phice = psc[srce::SC_PHICE];
  s.tauocx = psc[srce::SC_TAUOCX];
  s.tauocy = psc[srce::SC_TAUOCY];
  s.r.wnmean = psc[srce::SC_WNMEAN];
  s.fpi = psc[srce::SC_FPI];
  for (int j = 0; j < 4; ++j) s.whitecap[j] = wc[j];
  s.taubbl[0] = tb[0];
  s.taubbl[1] = tb[1];
  s.tauice[0] = ti[0];
  s.tauice[1] = ti[1];
  s.shave = 0;
}

WWB_PD void srce_psc_out(const SrceSh& s, float* psc, float* wc, float* tb, float* ti,
                         int* shave) {
  psc[srce::SC_USTAR] = s.r.ustar;
  psc[srce::SC_USTDIR] = s.r.usdir;
  psc[srce::SC_TAUWX] = s.tauwx;
  psc[srce::SC_TAUWY] = s.tauwy;
  psc[srce::SC_DTDYN] = s.dtdyn;
  psc[srce::SC_FCUT] = s.fcut;
  psc[srce::SC_TAUOX] = s.tauox;
  psc[srce::SC_TAUOY] = s.tauoy;
  psc[srce::SC_TAUWIX] = s.tauwix;
  psc[srce::SC_TAUWIY] = s.tauwiy;
  psc[srce::SC_TAUWNX] = s.tauwnx;
  psc[srce::SC_TAUWNY] = s.tauwny;
  psc[srce::SC_PHIAW] = s.phiaw;
  psc[srce::SC_CHARN] = s.r.charn;
  psc[srce::SC_TWS] = s.tws;
  psc[srce::SC_PHIOC] = s.phioc;
  psc[srce::SC_PHIBBL] = s.phibbl;
  psc[srce::SC_PHICE] = s.phice;
  psc[srce::SC_TAUOCX] = s.tauocx;
  psc[srce::SC_TAUOCY] = s.tauocy;
  psc[srce::SC_WNMEAN] = s.r.wnmean;
  psc[srce::SC_FPI] = s.fpi;
  for (int j = 0; j < 4; ++j) wc[j] = s.whitecap[j];
  tb[0] = s.taubbl[0];
  tb[1] = s.taubbl[1];
  ti[0] = s.tauice[0];
  ti[1] = s.tauice[1];
  *shave = s.shave;
}

/// W3SRCE for one point: init, steps until done, finish.
WWB_PD void srce_point(const Cta& cta, const SrceCtx& x) {
  srce_init(cta, x);
  for (int guard = 0; guard < 100000; ++guard) {
    srce_step_a(cta, x);
    srce_dia(cta, x);
    srce_step_c(cta, x);
    if (x.sh->done) break;
  }
  srce_finish(cta, x);
}

}  // namespace pt
}  // namespace wwb
