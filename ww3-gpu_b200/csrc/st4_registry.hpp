// ww3-gpu_b200/csrc/st4_registry.hpp
// Host side of ww_st4_init / ww_st4_set_real / ww_st4_set_int / ww_st4_commit: the registered
// scalars and arrays of a grid and of the process (module arrays), their validation, and the
// ST4 Fields they make. Shared by the C ABI (which then copies the arrays to the device) and the
// host build of the kernels' source used by the CPU tests.
//
// Reference: ww3-gpu kokkos/src/fortran_iface/st4_shim.cpp:132-250 (registration: rank, lower
// bound and type checks, copy of the caller's array, module arrays one per process, last
// registration wins; check_arrays: the extents each array needs given the scalars, larger
// registrations accepted), :472-584 (init, set, commit status codes).
#pragma once

#include <string>
#include <vector>

#include "st4_params.hpp"
#include "st4_point.cuh"

namespace wwb {
namespace st4 {

/// One registered array: values (float or int) and extents.
struct Reg {
  std::vector<float> f;
  std::vector<int> i;
  std::vector<int> ext;
  bool set() const { return !ext.empty(); }
  long long size() const {
    long long n = 1;
    for (int e : ext) n *= e;
    return ext.empty() ? 0 : n;
  }
};

struct GridReg {
  Params p{};
  bool configured = false;
  Reg a[NARRAYS];  ///< grid arrays (module ids unused here)
};

struct ModuleReg {
  Reg a[NARRAYS];  ///< module arrays (TAUT, TAUHFT, TAUHFT2, FWTABLE)
  float delust = 0, delalp = 0, deltauw = 0, delu = 0, deltail = 0, delab = 0;
};

/// Stores one registration; returns a WwKokkosStatus value (0 OK, 6 TABLE).
inline int reg_set(GridReg& g, ModuleReg& m, int id, const void* data, bool is_int, int rank,
                   const int* lbound, const int* extent, std::string& why) {
  if (id < 0 || id >= NARRAYS || data == nullptr || lbound == nullptr || extent == nullptr) {
    why = "bad array id or null pointer";
    return 6;
  }
  const ArraySpec& s = kArraySpecs[id];
  if (s.is_int != is_int || s.rank != rank) {
    why = std::string("type or rank of ") + s.name;
    return 6;
  }
  for (int r = 0; r < rank; ++r) {
    if (lbound[r] != s.lbound || extent[r] <= 0) {
      why = std::string("LBOUND or extent of ") + s.name;
      return 6;
    }
  }
  Reg& dst = s.module ? m.a[id] : g.a[id];
  dst.ext.assign(extent, extent + rank);
  const long long n = dst.size();
  if (is_int) {
    dst.i.assign(static_cast<const int*>(data), static_cast<const int*>(data) + n);
    dst.f.clear();
  } else {
    dst.f.assign(static_cast<const float*>(data), static_cast<const float*>(data) + n);
    dst.i.clear();
  }
  return 0;
}

/// The extents ST4 needs of each array (a registration may be larger, never smaller).
inline bool reg_check(const GridReg& g, const ModuleReg& m, std::string& why) {
  const Params& p = g.p;
  const int sdsnth = p.mth / 2 - 1;
  auto need = [&](const Reg& r, const char* name, int e0, int e1 = 0, int e2 = 0,
                  bool exact = false) {
    if (!r.set()) {
      why = std::string(name) + " is not registered";
      return false;
    }
    const int e[3] = {e0, e1, e2};
    for (size_t k = 0; k < r.ext.size(); ++k) {
      if (exact ? r.ext[k] != e[k] : r.ext[k] < e[k]) {
        why = std::string(name) + " has the wrong shape";
        return false;
      }
    }
    return true;
  };
  const int nk = p.nk, nth = p.nth, nspec = p.nspec;
  bool ok = need(g.a[A_SIG], "SIG", nk + 2) && need(g.a[A_SIG2], "SIG2", nspec) &&
            need(g.a[A_DSIP], "DSIP", nk + 2) && need(g.a[A_DDEN], "DDEN", nk) &&
            need(g.a[A_DDEN2], "DDEN2", nspec) && need(g.a[A_ESIN], "ESIN", nspec + nth) &&
            need(g.a[A_ECOS], "ECOS", nspec + nth) && need(g.a[A_TH], "TH", nth) &&
            need(g.a[A_SATWEIGHTS], "SATWEIGHTS", 2 * sdsnth + 1, p.mth, 0, true) &&
            need(g.a[A_SATINDICES], "SATINDICES", 2 * sdsnth + 1, p.mth, 0, true) &&
            need(g.a[A_CUMULW], "CUMULW", p.mspec, p.mspec, 0, true) &&
            need(g.a[A_DCKI], "DCKI", kNkhs, kNkd, 0, true) &&
            need(g.a[A_QBI], "QBI", kNkhs, kNkd, 0, true) &&
            need(g.a[A_IKTAB], "IKTAB", p.mk, kNdtab, 0, true) &&
            need(m.a[A_FWTABLE], "FWTABLE", kSizeFwTable + 1, 0, 0, true);
  if (ok && p.sintailpar[0] > 0.5f) {
    ok = need(m.a[A_TAUT], "TAUT", kItauMax + 1, kJuMax + 1, 0, true) &&
         need(m.a[A_TAUHFT], "TAUHFT", kIustar + 1, kIalpha + 1, 0, true);
    if (ok && p.ttauwshelter > 0)
      ok = need(m.a[A_TAUHFT2], "TAUHFT2", kIustar + 1, kIalpha + 1, kIlevTail + 1, true);
  }
  return ok;
}

/// The grid's scalars with the module's DEL* merged in (the module state current at the call).
inline Params current_params(const GridReg& g, const ModuleReg& m) {
  Params p = g.p;
  p.delust = m.delust;
  p.delalp = m.delalp;
  p.deltauw = m.deltauw;
  p.delu = m.delu;
  p.deltail = m.deltail;
  p.delab = m.delab;
  return p;
}

/// SATWEIGHTS and SATINDICES transposed to (MTH, NSAT), so the direction index runs fastest.
inline void transpose_sat(const GridReg& g, std::vector<float>& w_t, std::vector<int>& i_t) {
  const Reg& w = g.a[A_SATWEIGHTS];
  const Reg& x = g.a[A_SATINDICES];
  const int nsat = w.ext[0], mth = w.ext[1];
  w_t.assign(static_cast<size_t>(nsat) * mth, 0.0f);
  i_t.assign(static_cast<size_t>(nsat) * mth, 1);
  for (int j = 0; j < nsat; ++j)
    for (int ith = 0; ith < mth; ++ith) {
      w_t[ith + static_cast<size_t>(j) * mth] = w.f[j + static_cast<size_t>(ith) * nsat];
      i_t[ith + static_cast<size_t>(j) * mth] = x.i[j + static_cast<size_t>(ith) * nsat];
    }
}

/// CUMULW transposed (MSPEC x MSPEC, square): W3SDS4's cumulative term walks rows IS2 for
/// consecutive IS, which the transpose makes contiguous.
inline void transpose_cumulw(const GridReg& g, std::vector<float>& t) {
  const Reg& c = g.a[A_CUMULW];
  const size_t n = c.ext[0];
  t.assign(n * n, 0.0f);
  for (size_t j = 0; j < n; ++j)
    for (size_t i = 0; i < n; ++i) t[j + i * n] = c.f[i + j * n];
}

/// Fields over host-resident copies (the CPU build of the kernels) or over device copies whose
/// pointers the caller fills in the same order (abi_st4.cpp).
struct FieldPtrs {
  const float *sig, *sig2, *dsip, *dden, *dden2, *esin, *ecos, *th, *satw_t, *cumulw_t, *dcki,
      *qbi, *taut, *tauhft, *tauhft2, *fwtable;
  const int *sati_t, *iktab;
};

inline pt::Fields make_fields(const GridReg& g, const FieldPtrs& q) {
  pt::Fields f{};
  f.sig = q.sig;
  f.sig2 = q.sig2;
  f.dsip = q.dsip;
  f.dden = q.dden;
  f.dden2 = q.dden2;
  f.esin = q.esin;
  f.ecos = q.ecos;
  f.th = q.th;
  f.satw_t = q.satw_t;
  f.sati_t = q.sati_t;
  f.nsat = g.a[A_SATWEIGHTS].ext[0];
  f.sat_ld = g.a[A_SATWEIGHTS].ext[1];
  f.cumulw = q.cumulw_t;
  f.cumulw_ld = g.a[A_CUMULW].ext[0];
  f.dcki = q.dcki;
  f.qbi = q.qbi;
  f.iktab = q.iktab;
  f.iktab_ld = g.a[A_IKTAB].ext[0];
  f.taut = q.taut;
  f.tauhft = q.tauhft;
  f.tauhft2 = q.tauhft2;
  f.fwtable = q.fwtable;
  return f;
}

}  // namespace st4
}  // namespace wwb
