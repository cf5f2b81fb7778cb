// ww3-gpu_b200/csrc/snl1_tables.hpp
// INSNL1 on the host: the DIA's quadruplet geometry, interpolation weights and AF11, plus the
// row-shift form the B200 kernel addresses instead of the 32 index tables.
//
// Reference: ww3-gpu kokkos/src/ww_kokkos/snl1_tables.cpp:82-329 (WW3 w3snl1md.F90 INSNL1,
// lines 483-786). The arithmetic (float32, INT truncation, the x**n chains) is the same
// because the tables must be bit-identical; the layout is this library's own.
//
// Row-shift form. Every index entry of INSNL1 is IT_n(ITH) + (IF_m(IFR) - 1) * NTH for one of
// eight wrapped direction shifts IT_n and eight frequency maps IF_m
// (snl1_tables.cpp:167-223). In 0-based scratch slots (entry + NTH) that is
// row * NTH + wrap(ith0 + shift_n) with row = IF_m(IFR), row 0 being the zero bins. The kernel
// keeps the spectrum and the eight interaction arrays as (rows x NTH) matrices in shared
// memory and computes the row and the wrapped column itself, so it reads no index table.
#pragma once

#include <cstdint>
#include <vector>

namespace wwb {

/// W3GDATMD's DIA scalars (ww_snl1_init's arguments).
struct Snl1Config {
  int nk, nth;
  float xfr, dth, lam, snlc1, kdcon, kdmn, snls1, snls2, snls3, fachfe;
  int nspec() const { return nk * nth; }
};

/// (ITn, IFm) of each stored table, 1-based n and m, in the order of the C ABI:
/// IP11..IP14, IM11..IM14, IP21..IP24, IM21..IM24 (snl1_tables.cpp:186-203) ...
inline constexpr int kPmMap[16][2] = {{2, 2}, {1, 2}, {2, 1}, {1, 1}, {8, 4}, {7, 4},
                                      {8, 3}, {7, 3}, {6, 2}, {5, 2}, {6, 1}, {5, 1},
                                      {4, 4}, {3, 4}, {4, 3}, {3, 3}};
/// ... and IC11, IC21 .. IC81, IC12, IC22 .. IC82 (snl1_tables.cpp:206-223).
inline constexpr int kIcMap[16][2] = {{6, 6}, {5, 6}, {6, 5}, {5, 5}, {4, 8}, {3, 8},
                                      {4, 7}, {3, 7}, {2, 6}, {1, 6}, {2, 5}, {1, 5},
                                      {8, 8}, {7, 8}, {8, 7}, {7, 7}};

struct Snl1Tables {
  int nfr = 0, nfrhgh = 0, nfrchg = 0, nspecx = 0, nspecy = 0, nspec = 0, nth = 0;
  float dal1 = 0, dal2 = 0, dal3 = 0;
  float awg[8] = {}, swg[8] = {};
  std::vector<int> ipim;   ///< 16 x NSPECX, 0-based entries
  std::vector<int> ic;     ///< 16 x NSPEC, 0-based entries
  std::vector<float> af11; ///< NSPECX
  // Row-shift form, valid when rowshift is true.
  bool rowshift = false;
  int shift[8] = {};       ///< IT_n(ITH) - ITH before wrapping, n = 1..8
  int ifrp = 0, ifrm = 0;  ///< IF1(IFR) = IFR + IFRP, IF3(IFR) = MAX(0, IFR + IFRM)
  std::vector<int> ifrow;  ///< 8 x NFRCHG: IF_m(IFR), m = 1..8, IFR = 1..NFRCHG
  std::vector<float> af11_row;  ///< NFRCHG: AF11 of each row (constant along a row)
};

/// INSNL1 from the configuration and SIG(1:NK). AF11 = x**11 is multiplied out by GCC's -O3
/// power tree, x^5 * x^6, as the gfortran -O3 build of WW3 does (snl1_tables.cpp:45-59).
/// Returns false when the configuration gives no extended spectrum.
bool build_snl1_tables(const Snl1Config& c, const float* sig, Snl1Tables& t);

/// Fills the row-shift form from the geometry of `c` and checks that it reproduces every index
/// entry of `t` (which may come from the caller). Also checks AF11 is constant along rows.
void derive_rowshift(const Snl1Config& c, Snl1Tables& t);

/// INSNL1's weights in double precision for the FP64 DIA: the same steps as the float tables
/// with every real in double (the FP64 restatement of W3SNL1 that surrogate errors are measured
/// against). af11 has one value per row (NFRCHG). Returns false when the double geometry's
/// integer offsets differ from the float tables' (the index tables would then differ too).
struct Snl1WeightsF64 {
  double dal1 = 0, dal2 = 0, dal3 = 0, awg[8] = {}, swg[8] = {};
  std::vector<double> af11_row;
};
bool build_snl1_weights_f64(const Snl1Config& c, const float* sig, const Snl1Tables& t,
                            Snl1WeightsF64& w);

}  // namespace wwb
