// ww3-gpu_b200/csrc/outg_kernel.cuh
// W3OUTG on the device (outg_kernel.cu): the gridded output parameters of every sea point from
// the resident spectrum VA, and the partition fields from W3CPRT's table.
// Reference: ww3-gpu kokkos/src/ww_kokkos/iogo_w3outg.hpp:150-763 and
// kokkos/src/fortran_iface/outg_c.hpp (the field order and packets).
#pragma once

#include <cuda_runtime.h>

namespace wwb {

/// The 46 fields of ww_outg_va in the order of outg_c.hpp's WwOutgField: 40 of (NFLD), then
/// EF, TH1M, STH1M, TH2M, STH2M (NFLD, E3DF(2,k):E3DF(3,k)) and P2SMS (NFLD, P2MSF(2):P2MSF(3)).
constexpr int kOutgN1d = 40;
constexpr int kOutgNField = 46;
enum OutgField {
  OG_HS = 0, OG_WLM, OG_T02, OG_T0M1, OG_T01, OG_FP0, OG_THM, OG_THS, OG_THP0, OG_HSIG, OG_QKK,
  OG_QP, OG_WBT, OG_STMAXE, OG_STMAXD, OG_HCMAXE, OG_HMAXE, OG_HCMAXD, OG_HMAXD, OG_ABA, OG_ABD,
  OG_UBA, OG_UBD, OG_SXX, OG_SYY, OG_SXY, OG_USSX, OG_USSY, OG_TUSX, OG_TUSY, OG_MSSX, OG_MSSY,
  OG_MSSD, OG_MSCX, OG_MSCY, OG_MSCD, OG_PRMS, OG_TPMS, OG_BHD, OG_CGE,
  OG_EF = kOutgN1d, OG_TH1M, OG_STH1M, OG_TH2M, OG_STH2M, OG_P2SMS
};

/// The scalars and device arrays of one W3OUTG call.
struct OutgArgs {
  int nk, nth, nseal, nsea, nx, ny, nfld, nspec;
  float dth, xfr, fte, ftwl, fttr, undef, stexu, steyu, stedu;
  int p2msf2, p2msf3, e3df2[5], e3df3[5];
  int ompg;
  int f3[5];  ///< FLOLOC(3,1:5): EF, TH1M, STH1M, TH2M, STH2M
  int f69;    ///< FLOLOC(6,9): P2SMS
  int ste;    ///< the space-time extremes: (STEXU > 0 and STEYU > 0) or STEDU > 0
  const float* va;  ///< VA(NSPEC, 0:NSEALM): point JSEA is column JSEA
  const float *cg, *wn;   ///< (0:NK+1, 0:NSEA)
  const float *dw, *sig;  ///< DW(0:NSEA), SIG(0:NK+1)
  const float *dden, *dsii;  ///< (NK)
  const float *ecos, *esin, *ec2, *es2, *esc;  ///< (NTH)
  const int *mapsf, *mapsta;  ///< MAPSF(NSEA,3), MAPSTA(NY,NX)
  float* ebd;                 ///< work EBD(NK, NSEAL)
  float* f[kOutgNField];      ///< the fields (2-D ones null when not allocated)
};

/// Sections 1-4 and the space-time extremes of W3OUTG for points 1..nseal, on device arrays.
void launch_outg(const OutgArgs& a, cudaStream_t s);

/// Section 6 (the partition fields), on device arrays: icprt (NICP,2), dtprt (DIMP, NDTP);
/// fields[0..14] (NROW, 0:NOSWLL), fields[15] PWST, fields[16] PNR (NROW).
struct OutgPartArgs {
  int nseal, nsea, nx, ny, nrow, noswll, nicp, ndtp, dimp;
  float undef, wscut;
  const int *mapsf, *mapsta, *icprt;
  const float* dtprt;
  float* f[17];
};
void launch_outg_part(const OutgPartArgs& a, cudaStream_t s);

}  // namespace wwb
