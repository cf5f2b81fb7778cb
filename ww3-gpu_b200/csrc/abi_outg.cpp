// ww3-gpu_b200/csrc/abi_outg.cpp
// The C ABI of W3OUTG on the device: ww_outg_va (sections 1-4 and the space-time extremes on the
// resident VA) and ww_outg_part (section 6, the partition fields from W3CPRT's table).
//
// Reference: ww3-gpu kokkos/src/fortran_iface/outg_c.hpp:12-125 (the packets, the field order and
// the status codes) and outg_shim.cpp:238-546 (what each entry checks, what it copies in, and
// which fields come back). The device path of the reference is the one kept: the inputs are
// copied in per call, the fields are device buffers kept between calls, and only the fields a
// host reader needs come back to WW3's arrays (the FLOGRD entries W3IOGO writes under FLOUTG,
// the FLOGR2 ones under FLOUTG2, and the FLOGRR ones W3IORS ('HOT') writes when OARST); a field
// not wanted keeps its host bits. VA is read on the device (va_device): it crosses only when the
// host holds the newer bits, and W3OUTG never writes it.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>

#include "outg_kernel.cuh"
#include "staging.hpp"
#include "step.hpp"
#include "va.hpp"
#include "wwb_common.hpp"

namespace wwb {
namespace {

Status g_outg;
int fail(int code, const char* what) { return g_outg.fail(code, what); }

Staging& staging() {
  static auto* s = new Staging();
  return *s;
}

// The packets of outg_c.hpp:12-47 and :74-104.
enum : int {
  kNk = 0, kNth, kNseal, kNsea, kNx, kNy, kNfld, kNogrp, kNgrpp, kFloutg, kFloutg2, kOarst,
  kOmpg, kP2msf2, kP2msf3, kE3df2, kE3df3 = kE3df2 + 5, kNIpar = kE3df3 + 5
};
enum : int {
  kDth = 0, kXfr, kFte, kFtwl, kFttr, kUndef, kStexu, kSteyu, kStedu, kWscut, kNRpar
};
enum : int {
  kPNseal = 0, kPNsea, kPNx, kPNy, kPNrow, kPNoswll, kPNicp, kPNdtp, kPDimp, kPNogrp, kPNgrpp,
  kPFloutg, kPFloutg2, kPNIpar
};
constexpr int kPNRpar = 2, kPN2d = 15, kPNField = 17;

// The (group, index) entries of FLOGRD that make W3IOGO ('WRITE') write each field, and of
// FLOGRR that make W3IORS ('HOT') write it (outg_shim.cpp:94-150, from w3iogomd.F90 and
// w3iorsmd.F90 at the reference's pin); {0, 0} ends a list. FP0 is written for (2,6) and (2,18).
struct Key {
  int i, j;
};
struct FieldKeys {
  Key grd[3];
  Key grr[2];
};
constexpr FieldKeys kKeys[kOutgNField] = {
    {{{2, 1}}, {{2, 1}}},           // HS
    {{{2, 2}}, {{2, 2}}},           // WLM
    {{{2, 3}}, {}},                 // T02
    {{{2, 4}}, {{2, 4}}},           // T0M1
    {{{2, 5}}, {{2, 5}}},           // T01
    {{{2, 6}, {2, 18}}, {{2, 6}}},  // FP0
    {{{2, 7}}, {{2, 7}}},           // THM
    {{{2, 8}}, {}},                 // THS
    {{{2, 9}}, {}},                 // THP0
    {{{2, 10}}, {}},                // HSIG
    {{{8, 6}}, {}},                 // QKK
    {{{8, 5}}, {}},                 // QP
    {{{2, 17}}, {}},                // WBT
    {{{2, 11}}, {}},                // STMAXE
    {{{2, 12}}, {}},                // STMAXD
    {{{2, 14}}, {}},                // HCMAXE
    {{{2, 13}}, {}},                // HMAXE
    {{{2, 16}}, {}},                // HCMAXD
    {{{2, 15}}, {}},                // HMAXD
    {{{7, 1}}, {}},                 // ABA
    {{{7, 1}}, {}},                 // ABD
    {{{7, 2}}, {{7, 2}}},           // UBA
    {{{7, 2}}, {{7, 2}}},           // UBD
    {{{6, 1}}, {}},                 // SXX
    {{{6, 1}}, {}},                 // SYY
    {{{6, 1}}, {}},                 // SXY
    {{{6, 6}}, {{6, 6}}},           // USSX
    {{{6, 6}}, {{6, 6}}},           // USSY
    {{{6, 5}}, {{6, 5}}},           // TUSX
    {{{6, 5}}, {{6, 5}}},           // TUSY
    {{{8, 1}}, {}},                 // MSSX
    {{{8, 1}}, {}},                 // MSSY
    {{{8, 3}}, {}},                 // MSSD
    {{{8, 2}}, {}},                 // MSCX
    {{{8, 2}}, {}},                 // MSCY
    {{{8, 4}}, {}},                 // MSCD
    {{{6, 7}}, {}},                 // PRMS
    {{{6, 7}}, {}},                 // TPMS
    {{{6, 3}}, {{6, 3}}},           // BHD
    {{{5, 3}}, {}},                 // CGE
    {{{3, 1}}, {}},                 // EF
    {{{3, 2}}, {}},                 // TH1M
    {{{3, 3}}, {}},                 // STH1M
    {{{3, 4}}, {}},                 // TH2M
    {{{3, 5}}, {}},                 // STH2M
    {{{6, 9}}, {}},                 // P2SMS
};

/// WW_KOKKOS_OUTG_COUNT=1: the calls, sea points and fields and bytes copied back, at exit
/// (outg_shim.cpp:152-175, :453-466).
std::atomic<long long> g_calls{0}, g_points{0}, g_back{0}, g_back_bytes{0};
std::atomic<long long> g_part_calls{0}, g_part_back{0}, g_part_back_bytes{0};
void print_counts() {
  std::fprintf(stderr, "ww_kokkos: W3OUTG Kokkos calls: %lld\n", g_calls.load());
  std::fprintf(stderr, "ww_kokkos: W3OUTG sea points: %lld\n", g_points.load());
  std::fprintf(stderr, "ww_kokkos: W3OUTG fields copied back D2H: %lld\n", g_back.load());
  std::fprintf(stderr, "ww_kokkos: W3OUTG bytes copied back D2H: %lld\n", g_back_bytes.load());
  std::fprintf(stderr, "ww_kokkos: W3OUTG partition-field Kokkos calls: %lld\n",
               g_part_calls.load());
  std::fprintf(stderr, "ww_kokkos: W3OUTG partition fields copied back D2H: %lld\n",
               g_part_back.load());
  std::fprintf(stderr, "ww_kokkos: W3OUTG partition bytes copied back D2H: %lld\n",
               g_part_back_bytes.load());
}
[[maybe_unused]] const bool g_count_on = [] {
  const char* v = std::getenv("WW_KOKKOS_OUTG_COUNT");
  const bool c = v != nullptr && std::strcmp(v, "1") == 0;
  if (c) std::atexit(print_counts);
  return c;
}();

template <class F>
int guarded(F&& f) {
  try {
    return f();
  } catch (const std::bad_alloc& e) {
    return fail(WW_KOKKOS_ERR_RUNTIME, e.what());
  } catch (const std::exception& e) {
    return fail(WW_KOKKOS_ERR_KERNEL, e.what());
  }
}

/// Every point 1..nseal must name a cell of the grid: the kernels index MAPSTA with it.
bool mapsf_ok(const int* mapsf, int nsea, int nseal, int nx, int ny) {
  for (int i = 0; i < nseal; ++i) {
    const int ix = mapsf[i], iy = mapsf[nsea + i];
    if (ix < 1 || ix > nx || iy < 1 || iy > ny) return false;
  }
  return true;
}

/// The packets of one W3OUTG call, checked: the kernel's scalars and flags, the extents of the
/// 2-D fields, and FLOLOC. Returns OK or the status (message prefixed by `who`).
struct OutgCall {
  OutgArgs a{};
  size_t n2[kOutgNField - kOutgN1d] = {};
  bool floutg = false, floutg2 = false, oarst = false;
  int nogrp = 0, ngrpp = 0;
  const int *flogrd = nullptr, *flogr2 = nullptr;
  /// FLOGRD(NOGRP,NGRPP), LOGICAL(4); an index past NGRPP is never set.
  bool lgrd(const int* f, int i, int j) const {
    return j <= ngrpp && f[(i - 1) + (j - 1) * nogrp] != 0;
  }
  bool floloc(int i, int j) const {
    return (floutg && lgrd(flogrd, i, j)) || (floutg2 && lgrd(flogr2, i, j));
  }
};

int outg_packets(const int* ipar, const float* rpar, const int* flogrd, const int* flogr2,
                 int nspec, int nsealm, float* const* fields, const char* who, OutgCall& c) {
  char msg[128];
  const auto bad = [&](int code, const char* what) {
    std::snprintf(msg, sizeof msg, "%s: %s", who, what);
    return fail(code, msg);
  };
  const int nk = ipar[kNk], nth = ipar[kNth], nseal = ipar[kNseal], nsea = ipar[kNsea];
  const int nx = ipar[kNx], ny = ipar[kNy], nfld = ipar[kNfld];
  c.nogrp = ipar[kNogrp];
  c.ngrpp = ipar[kNgrpp];
  if (nk < 1 || nth < 1 || nspec != nk * nth || nseal < 0 || nseal > nsealm || nsea < nseal ||
      nx < 1 || ny < 1 || nfld < nseal || c.nogrp < 10 || c.ngrpp < 1)
    return bad(WW_KOKKOS_ERR_BAD_SHAPE, "bad sizes");
  for (int k = 0; k < kOutgN1d; ++k)
    if (fields[k] == nullptr) return bad(WW_KOKKOS_ERR_BAD_SHAPE, "a null 1-D field");
  OutgArgs& a = c.a;
  a.nk = nk;
  a.nth = nth;
  a.nseal = nseal;
  a.nsea = nsea;
  a.nx = nx;
  a.ny = ny;
  a.nfld = nfld;
  a.nspec = nspec;
  a.dth = rpar[kDth];
  a.xfr = rpar[kXfr];
  a.fte = rpar[kFte];
  a.ftwl = rpar[kFtwl];
  a.fttr = rpar[kFttr];
  a.undef = rpar[kUndef];
  a.stexu = rpar[kStexu];
  a.steyu = rpar[kSteyu];
  a.stedu = rpar[kStedu];
  a.p2msf2 = ipar[kP2msf2];
  a.p2msf3 = ipar[kP2msf3];
  for (int k = 0; k < 5; ++k) {
    a.e3df2[k] = ipar[kE3df2 + k];
    a.e3df3[k] = ipar[kE3df3 + k];
  }
  a.ompg = ipar[kOmpg] != 0;
  c.floutg = ipar[kFloutg] != 0;
  c.floutg2 = ipar[kFloutg2] != 0;
  c.oarst = ipar[kOarst] != 0;
  c.flogrd = flogrd;
  c.flogr2 = flogr2;
  // The fields the caller leaves to the Fortran W3OUTG: CALC_U3STOKES, SKEWNESS, CALC_WBT.
  if (c.floloc(6, 8) || c.floloc(6, 12) || c.floloc(8, 7) || c.floloc(8, 8) ||
      c.floloc(8, 9) || c.floloc(2, 17))
    return bad(WW_KOKKOS_ERR_UNSUPPORTED, "a field left to the Fortran W3OUTG is requested");
  for (int k = 0; k < 5; ++k) {
    a.f3[k] = c.floloc(3, k + 1);
    c.n2[k] = a.e3df3[k] >= a.e3df2[k] ? static_cast<size_t>(a.e3df3[k] - a.e3df2[k] + 1) : 0;
    if (a.f3[k] && (fields[OG_EF + k] == nullptr || c.n2[k] == 0))
      return bad(WW_KOKKOS_ERR_BAD_SHAPE, "a requested 3-D field is not allocated");
  }
  a.f69 = c.floloc(6, 9);
  c.n2[5] = a.p2msf3 >= a.p2msf2 ? static_cast<size_t>(a.p2msf3 - a.p2msf2 + 1) : 0;
  if (a.f69 && (fields[OG_P2SMS] == nullptr || c.n2[5] == 0))
    return bad(WW_KOKKOS_ERR_BAD_SHAPE, "P2SMS is requested and not allocated");
  a.ste = (a.stexu > 0.0f && a.steyu > 0.0f) || a.stedu > 0.0f;
  return WW_KOKKOS_OK;
}

int run_outg(int igrid, const int* ipar, const float* rpar, const int* flogrd, const int* flogr2,
             const int* flogrr, float* va, int nspec, int nsealm, const float* cg,
             const float* wn, const float* dw, const float* sig, const float* dden,
             const float* dsii, const float* ecos, const float* esin, const float* ec2,
             const float* es2, const float* esc, const int* mapsf, const int* mapsta,
             float* const* fields) {
  OutgCall c;
  const int prc = outg_packets(ipar, rpar, flogrd, flogr2, nspec, nsealm, fields, "ww_outg_va", c);
  if (prc != WW_KOKKOS_OK) return prc;
  OutgArgs& a = c.a;
  const int nk = a.nk, nth = a.nth, nseal = a.nseal, nsea = a.nsea, nx = a.nx, ny = a.ny;
  const int nfld = a.nfld;
  const size_t* n2 = c.n2;
  const bool oarst = c.oarst;
  const auto floloc = [&](int i, int j) { return c.floloc(i, j); };
  const auto lgrd = [&](const int* f, int i, int j) { return c.lgrd(f, i, j); };
  if (!mapsf_ok(mapsf, nsea, nseal, nx, ny))
    return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_outg_va: MAPSF names a cell outside the grid");
  if (!runtime().ready) return fail(WW_KOKKOS_ERR_NOT_INITIALISED, "before ww_kokkos_init");
  if (step_recorder(igrid) != nullptr)
    return fail(WW_KOKKOS_ERR_UNSUPPORTED, "ww_outg_va: the grid is recording a step");

  timers::Region t_call("outg.call");
  float* d_va = nullptr;
  const int rc = va_device(igrid, va, nspec, nsealm, &d_va);
  if (rc != WW_KOKKOS_OK) return fail(rc, "ww_outg_va: the resident VA refused this call");
  a.va = d_va;
  Staging& st = staging();
  cudaStream_t s = runtime().stream;
  const size_t nf = static_cast<size_t>(nfld);
  {
    timers::Region t("outg.h2d");
    const size_t nk2 = static_cast<size_t>(nk) + 2, ns1 = static_cast<size_t>(nsea) + 1;
    const size_t nt = static_cast<size_t>(nth);
    int slot = 0;
    a.cg = st.in(slot++, cg, nk2 * ns1, s);
    a.wn = st.in(slot++, wn, nk2 * ns1, s);
    a.dw = st.in(slot++, dw, ns1, s);
    a.sig = st.in(slot++, sig, nk2, s);
    a.dden = st.in(slot++, dden, static_cast<size_t>(nk), s);
    a.dsii = st.in(slot++, dsii, static_cast<size_t>(nk), s);
    a.ecos = st.in(slot++, ecos, nt, s);
    a.esin = st.in(slot++, esin, nt, s);
    a.ec2 = st.in(slot++, ec2, nt, s);
    a.es2 = st.in(slot++, es2, nt, s);
    a.esc = st.in(slot++, esc, nt, s);
    a.mapsf = st.in(slot++, mapsf, static_cast<size_t>(nsea) * 3, s);
    a.mapsta = st.in(slot++, mapsta, static_cast<size_t>(nx) * ny, s);
    a.ebd = static_cast<float*>(st.get(slot++, sizeof(float) * nk * static_cast<size_t>(nseal)));
    constexpr int kField0 = 20;
    for (int k = 0; k < kOutgN1d; ++k)
      a.f[k] = static_cast<float*>(st.get(kField0 + k, sizeof(float) * nf));
    for (int k = 0; k < kOutgNField - kOutgN1d; ++k) {
      const bool on = k < 5 ? a.f3[k] != 0 : a.f69 != 0;
      a.f[kOutgN1d + k] =
          on ? static_cast<float*>(st.get(kField0 + kOutgN1d + k, sizeof(float) * nf * n2[k]))
             : nullptr;
    }
    // W3OUTG writes CGE at sea points only: its device buffer starts from the host bits.
    WWB_CHECK(cudaMemcpyAsync(a.f[OG_CGE], fields[OG_CGE], sizeof(float) * nf,
                              cudaMemcpyHostToDevice, s));
  }
  {
    timers::Region t("outg.kernel");
    launch_outg(a, s);
  }
  {
    timers::Region t("outg.d2h");
    for (int k = 0; k < kOutgNField; ++k) {
      bool want = false;
      for (const Key& key : kKeys[k].grd)
        if (key.i != 0) want = want || floloc(key.i, key.j);
      if (oarst)
        for (const Key& key : kKeys[k].grr)
          if (key.i != 0) want = want || lgrd(flogrr, key.i, key.j);
      if (!want) continue;
      const size_t n = k < kOutgN1d ? nf : nf * n2[k - kOutgN1d];
      if (n == 0 || a.f[k] == nullptr || fields[k] == nullptr) continue;
      if (k < kOutgN1d) {
        WWB_CHECK(
            cudaMemcpyAsync(fields[k], a.f[k], sizeof(float) * n, cudaMemcpyDeviceToHost, s));
      } else if (nseal > 0) {
        // Section 1 does not reset the 2-D fields: rows past NSEAL, and the columns of an IK
        // outside 1..NK, keep the caller's bits; only the rows and columns written come back.
        const int lo = k < OG_P2SMS ? a.e3df2[k - kOutgN1d] : a.p2msf2;
        const long long c0 = lo < 1 ? 1 - lo : 0;
        const long long c1 = std::min<long long>(static_cast<long long>(n2[k - kOutgN1d]) - 1,
                                                 static_cast<long long>(nk) - lo);
        if (c1 >= c0)
          WWB_CHECK(cudaMemcpy2DAsync(fields[k] + c0 * nf, sizeof(float) * nf, a.f[k] + c0 * nf,
                                      sizeof(float) * nf, sizeof(float) * nseal,
                                      static_cast<size_t>(c1 - c0 + 1), cudaMemcpyDeviceToHost,
                                      s));
      }
      g_back.fetch_add(1, std::memory_order_relaxed);
      g_back_bytes.fetch_add(static_cast<long long>(n * sizeof(float)), std::memory_order_relaxed);
    }
    WWB_CHECK(cudaStreamSynchronize(s));
  }
  g_calls.fetch_add(1, std::memory_order_relaxed);
  g_points.fetch_add(nseal, std::memory_order_relaxed);
  g_outg.ok();
  return WW_KOKKOS_OK;
}

int run_outg_device(const int* ipar, const float* rpar, const int* flogrd, const int* flogr2,
                    const float* d_va, int nspec, int nsealm, const float* cg, const float* wn,
                    const float* dw, const float* sig, const float* dden, const float* dsii,
                    const float* ecos, const float* esin, const float* ec2, const float* es2,
                    const float* esc, const int* mapsf, const int* mapsta, float* ebd,
                    float* const* fields, void* stream) {
  OutgCall c;
  const int prc =
      outg_packets(ipar, rpar, flogrd, flogr2, nspec, nsealm, fields, "ww_outg_device", c);
  if (prc != WW_KOKKOS_OK) return prc;
  if (c.a.nseal > 0 && ebd == nullptr)
    return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_outg_device: a null EBD work array");
  if (!runtime().ready) return fail(WW_KOKKOS_ERR_NOT_INITIALISED, "before ww_kokkos_init");
  OutgArgs& a = c.a;
  a.va = d_va;
  a.cg = cg;
  a.wn = wn;
  a.dw = dw;
  a.sig = sig;
  a.dden = dden;
  a.dsii = dsii;
  a.ecos = ecos;
  a.esin = esin;
  a.ec2 = ec2;
  a.es2 = es2;
  a.esc = esc;
  a.mapsf = mapsf;
  a.mapsta = mapsta;
  a.ebd = ebd;
  for (int k = 0; k < kOutgNField; ++k) {
    const bool on = k < kOutgN1d || (k < OG_P2SMS ? a.f3[k - kOutgN1d] != 0 : a.f69 != 0);
    a.f[k] = on ? fields[k] : nullptr;
  }
  launch_outg(a, static_cast<cudaStream_t>(stream));
  g_calls.fetch_add(1, std::memory_order_relaxed);
  g_points.fetch_add(a.nseal, std::memory_order_relaxed);
  g_outg.ok();
  return WW_KOKKOS_OK;
}

int run_part(const int* ipar, const float* rpar, const int* flogrd, const int* flogr2,
             const int* mapsf, const int* mapsta, const int* icprt, const float* dtprt,
             float* const* fields) {
  const int nseal = ipar[kPNseal], nsea = ipar[kPNsea], nx = ipar[kPNx], ny = ipar[kPNy];
  const int nrow = ipar[kPNrow], noswll = ipar[kPNoswll], nicp = ipar[kPNicp];
  const int ndtp = ipar[kPNdtp], nogrp = ipar[kPNogrp], ngrpp = ipar[kPNgrpp];
  if (nseal < 0 || nsea < nseal || nx < 1 || ny < 1 || nrow < nseal || noswll < 0 ||
      nicp < nseal + 1 || ndtp < 1 || ipar[kPDimp] != 15 || nogrp < 4 || ngrpp < 17)
    return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_outg_part: bad sizes");
  for (int k = 0; k < kPNField; ++k)
    if (fields[k] == nullptr) return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_outg_part: a null field");
  if (!mapsf_ok(mapsf, nsea, nseal, nx, ny))
    return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_outg_part: MAPSF names a cell outside the grid");
  // The columns of DTPRT a sea point reads: N2 .. N2+N1-1 (its wind sea and swells).
  for (int j = 0; j < nseal; ++j) {
    const int ix = mapsf[j], iy = mapsf[nsea + j];
    if (mapsta[(ix - 1) * ny + (iy - 1)] <= 0) continue;
    const int n1 = icprt[j], n2 = icprt[nicp + j];
    if (n1 >= 1 && (n2 < 1 || static_cast<long long>(n2) + (n1 > 1 ? n1 - 1 : 0) > ndtp))
      return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_outg_part: ICPRT points outside DTPRT");
  }
  if (!runtime().ready) return fail(WW_KOKKOS_ERR_NOT_INITIALISED, "before ww_kokkos_init");
  const bool floutg = ipar[kPFloutg] != 0, floutg2 = ipar[kPFloutg2] != 0;
  const auto want = [&](int j) {
    const int k = 3 + (j - 1) * nogrp;  // FLOGRD(4,j)
    return (floutg && flogrd[k] != 0) || (floutg2 && flogr2[k] != 0);
  };

  timers::Region t_call("outg.part");
  Staging& st = staging();
  cudaStream_t s = runtime().stream;
  OutgPartArgs a{};
  a.nseal = nseal;
  a.nsea = nsea;
  a.nx = nx;
  a.ny = ny;
  a.nrow = nrow;
  a.noswll = noswll;
  a.nicp = nicp;
  a.ndtp = ndtp;
  a.dimp = 15;
  a.undef = rpar[0];
  a.wscut = rpar[1];
  constexpr int k0 = 100;
  a.mapsf = st.in(k0, mapsf, static_cast<size_t>(nsea) * 3, s);
  a.mapsta = st.in(k0 + 1, mapsta, static_cast<size_t>(nx) * ny, s);
  a.icprt = st.in(k0 + 2, icprt, static_cast<size_t>(nicp) * 2, s);
  a.dtprt = st.in(k0 + 3, dtprt, static_cast<size_t>(15) * ndtp, s);
  const size_t nr = static_cast<size_t>(nrow), nc = static_cast<size_t>(noswll) + 1;
  for (int k = 0; k < kPNField; ++k)
    a.f[k] = static_cast<float*>(st.get(k0 + 10 + k, sizeof(float) * (k < kPN2d ? nr * nc : nr)));
  launch_outg_part(a, s);
  for (int k = 0; k < kPNField; ++k) {
    if (!want(k + 1)) continue;
    const size_t n = k < kPN2d ? nr * nc : nr;
    if (n == 0) continue;
    WWB_CHECK(cudaMemcpyAsync(fields[k], a.f[k], sizeof(float) * n, cudaMemcpyDeviceToHost, s));
    g_part_back.fetch_add(1, std::memory_order_relaxed);
    g_part_back_bytes.fetch_add(static_cast<long long>(n * sizeof(float)),
                                std::memory_order_relaxed);
  }
  WWB_CHECK(cudaStreamSynchronize(s));
  g_part_calls.fetch_add(1, std::memory_order_relaxed);
  g_outg.ok();
  return WW_KOKKOS_OK;
}

}  // namespace

void release_outg_staging() { staging().release(); }

}  // namespace wwb

using namespace wwb;

extern "C" {

int ww_outg_va(int igrid, const int* ipar, int nipar, const float* rpar, int nrpar,
               const int* flogrd, const int* flogr2, const int* flogrr, float* va, int nspec,
               int nsealm, const float* cg, const float* wn, const float* dw, const float* sig,
               const float* dden, const float* dsii, const float* ecos, const float* esin,
               const float* ec2, const float* es2, const float* esc, const int* mapsf,
               const int* mapsta, float* const* fields, int nfields) {
  if (ipar == nullptr || rpar == nullptr || nipar != kNIpar || nrpar != kNRpar ||
      nfields != kOutgNField || fields == nullptr)
    return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_outg_va: bad packet");
  if (flogrd == nullptr || flogr2 == nullptr || flogrr == nullptr || va == nullptr ||
      cg == nullptr || wn == nullptr || dw == nullptr || sig == nullptr || dden == nullptr ||
      dsii == nullptr || ecos == nullptr || esin == nullptr || ec2 == nullptr || es2 == nullptr ||
      esc == nullptr || mapsf == nullptr || mapsta == nullptr)
    return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_outg_va: a null pointer");
  return guarded([&] {
    return run_outg(igrid, ipar, rpar, flogrd, flogr2, flogrr, va, nspec, nsealm, cg, wn, dw, sig,
                    dden, dsii, ecos, esin, ec2, es2, esc, mapsf, mapsta, fields);
  });
}

int ww_outg_device(const int* ipar, int nipar, const float* rpar, int nrpar, const int* flogrd,
                   const int* flogr2, const float* d_va, int nspec, int nsealm, const float* cg,
                   const float* wn, const float* dw, const float* sig, const float* dden,
                   const float* dsii, const float* ecos, const float* esin, const float* ec2,
                   const float* es2, const float* esc, const int* mapsf, const int* mapsta,
                   float* ebd, float* const* fields, int nfields, void* stream) {
  if (ipar == nullptr || rpar == nullptr || nipar != kNIpar || nrpar != kNRpar ||
      nfields != kOutgNField || fields == nullptr || flogrd == nullptr || flogr2 == nullptr)
    return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_outg_device: bad packet");
  if (d_va == nullptr || cg == nullptr || wn == nullptr || dw == nullptr || sig == nullptr ||
      dden == nullptr || dsii == nullptr || ecos == nullptr || esin == nullptr || ec2 == nullptr ||
      es2 == nullptr || esc == nullptr || mapsf == nullptr || mapsta == nullptr)
    return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_outg_device: a null pointer");
  return guarded([&] {
    return run_outg_device(ipar, rpar, flogrd, flogr2, d_va, nspec, nsealm, cg, wn, dw, sig,
                           dden, dsii, ecos, esin, ec2, es2, esc, mapsf, mapsta, ebd, fields,
                           stream);
  });
}

int ww_outg_part(const int* ipar, int nipar, const float* rpar, int nrpar, const int* flogrd,
                 const int* flogr2, const int* mapsf, const int* mapsta, const int* icprt,
                 const float* dtprt, float* const* fields, int nfields) {
  if (ipar == nullptr || rpar == nullptr || nipar != kPNIpar || nrpar != kPNRpar ||
      nfields != kPNField || fields == nullptr || flogrd == nullptr || flogr2 == nullptr ||
      mapsf == nullptr || mapsta == nullptr || icprt == nullptr || dtprt == nullptr)
    return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_outg_part: bad packet");
  return guarded(
      [&] { return run_part(ipar, rpar, flogrd, flogr2, mapsf, mapsta, icprt, dtprt, fields); });
}

int ww_outg_last_error(void) { return g_outg.get(); }

}  // extern "C"
