// ww3-gpu_b200/csrc/st4_params.hpp
// The ST4 source-term package's scalars as they cross the C ABI (RPAR/IPAR packets), the
// W3SRCE packets, and the array identifiers of ww_st4_set_real/int.
//
// The packet layout is the reference's interface, kept index for index so the same Fortran
// caller fills both: ww3-gpu kokkos/src/ww_kokkos/st4_params.hpp:79-154 (ST4 RPAR/IPAR),
// srce_params.hpp:36-84 (W3SRCE RPAR/IPAR), st4_arrays.hpp:41-81 (ArrayId, rank, lower bound,
// module or grid scope). The scalars are WAVEWATCH III's (w3src4md.F90, w3gdatmd.F90,
// constants.F90).
#pragma once

#include <cstdint>

namespace wwb {
namespace st4 {

// ---------------------------------------------------------------------------- ST4 RPAR / IPAR
enum Rpar : int {
  R_DTH = 0, R_XFR, R_FTE, R_FTF, R_AAIRCMIN, R_AAIRGB, R_IGPARS5, R_WWNMEANPTAIL,
  R_SSTXFTFTAIL, R_AALPHA, R_BBETA, R_ZZ0MAX, R_ZZ0RAT, R_ZZALP, R_SSINTHP, R_TTAUWSHELTER,
  R_SSWELLF,                 // SSWELLF(1:7)
  R_SSDSC = R_SSWELLF + 7,   // SSDSC(1:21)
  R_SSDSBR = R_SSDSC + 21,
  R_SINTAILPAR,              // SINTAILPAR(1:5)
  R_SSDSP = R_SINTAILPAR + 5,
  R_WWNMEANP, R_SSTXFTWN, R_SSDSBRF1, R_SSDSBINT, R_SSDSBCK, R_SSDSHCK, R_SSDSABK, R_SSDSPBK,
  R_CAPCHNK,                 // CAPCHNK(1:10)
  R_ZZWND = R_CAPCHNK + 10,
  R_SSDSCOS, R_SSDSDTH, R_SSDSBT,
  R_SSDSBM,                  // SSDSBM(0:4)
  R_DELUST = R_SSDSBM + 5,   // W3SRC4MD module scalars
  R_DELALP, R_DELTAUW, R_DELU, R_DELTAIL,
  R_DELAB,                   // CONSTANTS DELAB
  NRPAR
};

enum Ipar : int { I_NK = 0, I_NTH, I_NSPEC, I_MK, I_MTH, I_MSPEC, I_STAB3, I_IG1, I_FLX5, NIPAR };

/// The ST4 scalars, unpacked (WW3 names in lower case); a plain aggregate passed to kernels by
/// value.
struct Params {
  int nk, nth, nspec, mk, mth, mspec, stab3, ig1;
  float dth, xfr, fte, ftf, aaircmin, aairgb, igpars5, wwnmeanptail, sstxftftail;
  float aalpha, bbeta, zz0max, zz0rat, zzalp, ssinthp, ttauwshelter;
  float sswellf[7], ssdsc[21], ssdsbr, sintailpar[5], ssdsp, wwnmeanp, sstxftwn;
  float ssdsbrf1, ssdsbint, ssdsbck, ssdshck, ssdsabk, ssdspbk, capchnk[10];
  float zzwnd, ssdscos, ssdsdth, ssdsbt, ssdsbm[5];
  float delust, delalp, deltauw, delu, deltail, delab;
};

inline Params unpack(const float* r, const int* i) {
  Params p{};
  p.nk = i[I_NK];
  p.nth = i[I_NTH];
  p.nspec = i[I_NSPEC];
  p.mk = i[I_MK];
  p.mth = i[I_MTH];
  p.mspec = i[I_MSPEC];
  p.stab3 = i[I_STAB3];
  p.ig1 = i[I_IG1];
  p.dth = r[R_DTH];
  p.xfr = r[R_XFR];
  p.fte = r[R_FTE];
  p.ftf = r[R_FTF];
  p.aaircmin = r[R_AAIRCMIN];
  p.aairgb = r[R_AAIRGB];
  p.igpars5 = r[R_IGPARS5];
  p.wwnmeanptail = r[R_WWNMEANPTAIL];
  p.sstxftftail = r[R_SSTXFTFTAIL];
  p.aalpha = r[R_AALPHA];
  p.bbeta = r[R_BBETA];
  p.zz0max = r[R_ZZ0MAX];
  p.zz0rat = r[R_ZZ0RAT];
  p.zzalp = r[R_ZZALP];
  p.ssinthp = r[R_SSINTHP];
  p.ttauwshelter = r[R_TTAUWSHELTER];
  for (int j = 0; j < 7; ++j) p.sswellf[j] = r[R_SSWELLF + j];
  for (int j = 0; j < 21; ++j) p.ssdsc[j] = r[R_SSDSC + j];
  p.ssdsbr = r[R_SSDSBR];
  for (int j = 0; j < 5; ++j) p.sintailpar[j] = r[R_SINTAILPAR + j];
  p.ssdsp = r[R_SSDSP];
  p.wwnmeanp = r[R_WWNMEANP];
  p.sstxftwn = r[R_SSTXFTWN];
  p.ssdsbrf1 = r[R_SSDSBRF1];
  p.ssdsbint = r[R_SSDSBINT];
  p.ssdsbck = r[R_SSDSBCK];
  p.ssdshck = r[R_SSDSHCK];
  p.ssdsabk = r[R_SSDSABK];
  p.ssdspbk = r[R_SSDSPBK];
  for (int j = 0; j < 10; ++j) p.capchnk[j] = r[R_CAPCHNK + j];
  p.zzwnd = r[R_ZZWND];
  p.ssdscos = r[R_SSDSCOS];
  p.ssdsdth = r[R_SSDSDTH];
  p.ssdsbt = r[R_SSDSBT];
  for (int j = 0; j < 5; ++j) p.ssdsbm[j] = r[R_SSDSBM + j];
  p.delust = r[R_DELUST];
  p.delalp = r[R_DELALP];
  p.deltauw = r[R_DELTAUW];
  p.delu = r[R_DELU];
  p.deltail = r[R_DELTAIL];
  p.delab = r[R_DELAB];
  return p;
}

// ------------------------------------------------------------------------------ ST4 arrays
enum ArrayId : int {
  A_SIG = 0, A_SIG2, A_DSIP, A_DDEN, A_DDEN2, A_ESIN, A_ECOS, A_TH, A_SATWEIGHTS, A_CUMULW,
  A_DCKI, A_QBI, A_SATINDICES, A_IKTAB, A_TAUT, A_TAUHFT, A_TAUHFT2, A_FWTABLE, NARRAYS
};

struct ArraySpec {
  const char* name;
  bool is_int;
  int rank;
  int lbound;   ///< of every dimension
  bool module;  ///< one copy per process (W3SRC4MD / CONSTANTS module array): last one wins
};

inline constexpr ArraySpec kArraySpecs[NARRAYS] = {
    {"SIG", false, 1, 0, false},        {"SIG2", false, 1, 1, false},
    {"DSIP", false, 1, 0, false},       {"DDEN", false, 1, 1, false},
    {"DDEN2", false, 1, 1, false},      {"ESIN", false, 1, 1, false},
    {"ECOS", false, 1, 1, false},       {"TH", false, 1, 1, false},
    {"SATWEIGHTS", false, 2, 1, false}, {"CUMULW", false, 2, 1, false},
    {"DCKI", false, 2, 1, false},       {"QBI", false, 2, 1, false},
    {"SATINDICES", true, 2, 1, false},  {"IKTAB", true, 2, 1, false},
    {"TAUT", false, 2, 0, true},        {"TAUHFT", false, 2, 0, true},
    {"TAUHFT2", false, 3, 0, true},     {"FWTABLE", false, 1, 0, true},
};

// W3SRC4MD / W3GDATMD / CONSTANTS parameters the kernels use (w3src4md.F90:61-71,
// w3gdatmd.F90:637-638, constants.F90:92-95).
constexpr int kItauMax = 200, kJuMax = 200, kIustar = 100, kIalpha = 200, kIlevTail = 50;
constexpr int kNkhs = 2000, kNkd = 1300, kNdtab = 2000, kSizeFwTable = 300;

}  // namespace st4

namespace srce {

// ------------------------------------------------------------------------- W3SRCE RPAR / IPAR
enum Rpar : int {
  R_DMIN = 0, R_DTMAX, R_DTMIN, R_FACTI1, R_FACTI2, R_FACHFA, R_FACP, R_XFLT, R_XREL, R_FHMAX,
  R_FFXFM, R_FFXPM, R_FFXFA,
  R_ICESCALES,                // ICESCALES(1:4)
  R_SLNC1 = R_ICESCALES + 4,
  R_FSPM, R_FSHF, R_SBTC1, R_SDBC1, R_SDBC2, R_FACSD, R_FTTR, R_FLDALPHA, R_TAIL_LEV,
  R_TAIL_TRAN1, R_TAIL_TRAN2,
  NRPAR
};

enum Ipar : int {
  I_NK = 0, I_NTH, I_NSPEC, I_IQTPE, I_IICEDISP, I_IC_NUMERICS, I_FDONLY, I_LAB_SWITCH, I_LN1,
  I_SEED, I_FLD2, I_TAIL_ID, NIPAR
};

struct Params {
  int nk, nth, nspec, iqtpe, iicedisp, ic_numerics, fdonly, ln1, seed, fld2, tail_id;
  float dmin, dtmax, dtmin, facti1, facti2, fachfa, facp, xflt, xrel, fhmax, ffxfm, ffxpm, ffxfa;
  float icescales[4];
  float slnc1, fspm, fshf, sbtc1, sdbc1, sdbc2, facsd, fttr, fldalpha, tail_lev, tail_tran1,
      tail_tran2;
};

inline Params unpack(const float* r, const int* i) {
  Params p{};
  p.nk = i[I_NK];
  p.nth = i[I_NTH];
  p.nspec = i[I_NSPEC];
  p.iqtpe = i[I_IQTPE];
  p.iicedisp = i[I_IICEDISP];
  p.ic_numerics = i[I_IC_NUMERICS];
  p.fdonly = i[I_FDONLY];
  p.ln1 = i[I_LN1];
  p.seed = i[I_SEED];
  p.fld2 = i[I_FLD2];
  p.tail_id = i[I_TAIL_ID];
  p.dmin = r[R_DMIN];
  p.dtmax = r[R_DTMAX];
  p.dtmin = r[R_DTMIN];
  p.facti1 = r[R_FACTI1];
  p.facti2 = r[R_FACTI2];
  p.fachfa = r[R_FACHFA];
  p.facp = r[R_FACP];
  p.xflt = r[R_XFLT];
  p.xrel = r[R_XREL];
  p.fhmax = r[R_FHMAX];
  p.ffxfm = r[R_FFXFM];
  p.ffxpm = r[R_FFXPM];
  p.ffxfa = r[R_FFXFA];
  for (int j = 0; j < 4; ++j) p.icescales[j] = r[R_ICESCALES + j];
  p.slnc1 = r[R_SLNC1];
  p.fspm = r[R_FSPM];
  p.fshf = r[R_FSHF];
  p.sbtc1 = r[R_SBTC1];
  p.sdbc1 = r[R_SDBC1];
  p.sdbc2 = r[R_SDBC2];
  p.facsd = r[R_FACSD];
  p.fttr = r[R_FTTR];
  p.fldalpha = r[R_FLDALPHA];
  p.tail_lev = r[R_TAIL_LEV];
  p.tail_tran1 = r[R_TAIL_TRAN1];
  p.tail_tran2 = r[R_TAIL_TRAN2];
  return p;
}

/// Rows of ww_srce_batch's per-point packets (ww_kokkos_c.hpp:231-251, same order).
enum In : int { IN_D_INP = 0, IN_U10ABS, IN_U10DIR, IN_AS, IN_ICE, IN_DAIR, IN_COEF, NPIN };
enum Scal : int {
  SC_USTAR = 0, SC_USTDIR, SC_TAUWX, SC_TAUWY, SC_DTDYN, SC_FCUT, SC_TAUOX, SC_TAUOY, SC_TAUWIX,
  SC_TAUWIY, SC_TAUWNX, SC_TAUWNY, SC_PHIAW, SC_CHARN, SC_TWS, SC_PHIOC, SC_PHIBBL, SC_PHICE,
  SC_TAUOCX, SC_TAUOCY, SC_WNMEAN, SC_FPI, NPSC
};

}  // namespace srce
}  // namespace wwb
