// ww3-gpu_b200/csrc/snl1_tables.cpp
// INSNL1 on the host (see snl1_tables.hpp). Compiled with -ffp-contract=off: every float
// operation below rounds on its own, as in the gfortran build of WW3 and the reference's C++.
#include "snl1_tables.hpp"

#include <cmath>

namespace wwb {
namespace {

/// x**n for a runtime INTEGER n as gfortran evaluates it: libgcc's __powisf2 binary chain
/// (reference snl1_tables.cpp:26-43).
float powi(float x, int n) {
  unsigned m = n < 0 ? static_cast<unsigned>(-n) : static_cast<unsigned>(n);
  float y = (m & 1u) ? x : 1.0f;
  while ((m >>= 1u) != 0u) {
    x = x * x;
    if (m & 1u) y = y * x;
  }
  return n < 0 ? 1.0f / y : y;
}

/// x**11 by GCC's -O3 power tree: x2, x3 = x2*x, x5 = x2*x3, x6 = x3*x3, x11 = x5*x6.
float pow11(float x) {
  const float x2 = x * x;
  const float x3 = x2 * x;
  const float x5 = x2 * x3;
  const float x6 = x3 * x3;
  return x5 * x6;
}

/// The quadruplet geometry of sections 1-5 and 9 of INSNL1.
struct Geometry {
  int ithp, ithp1, ithm, ithm1, ifrp, ifrp1, ifrm, ifrm1;
  float dal1, dal2, dal3, awg[8];
};

Geometry geometry(const Snl1Config& c) {
  Geometry g{};
  const float one = 1.0f;
  // 1. Internal angles of the quadruplet.
  const float lamm2_b = one - c.lam, lamp2_b = one + c.lam;
  const float lamm2 = lamm2_b * lamm2_b, lamp2 = lamp2_b * lamp2_b;
  const float delth3 = std::acos((lamm2 * lamm2 + 4.0f - lamp2 * lamp2) / (4.0f * lamm2));
  const float delth4 = std::asin(-std::sin(delth3) * lamm2 / lamp2);
  // 2. Lambda-dependent weights: 1/(1+LAM)**4, 1/(1-LAM)**4.
  const float p2 = lamp2_b * lamp2_b, m2 = lamm2_b * lamm2_b;
  g.dal1 = one / (p2 * p2);
  g.dal2 = one / (m2 * m2);
  g.dal3 = 2.0f * g.dal1 * g.dal2;
  // 3. Directional indices and weights.
  const float cthp = std::fabs(delth4 / c.dth);
  g.ithp = static_cast<int>(cthp);
  g.ithp1 = g.ithp + 1;
  const float wthp = cthp - static_cast<float>(g.ithp), wthp1 = one - wthp;
  const float cthm = std::fabs(delth3 / c.dth);
  g.ithm = static_cast<int>(cthm);
  g.ithm1 = g.ithm + 1;
  const float wthm = cthm - static_cast<float>(g.ithm), wthm1 = one - wthm;
  // 4. Frequency indices and weights.
  const float xfrln = std::log(c.xfr);
  g.ifrp = static_cast<int>(std::log(one + c.lam) / xfrln);
  g.ifrp1 = g.ifrp + 1;
  const float wfrp = (one + c.lam - powi(c.xfr, g.ifrp)) /
                     (powi(c.xfr, g.ifrp1) - powi(c.xfr, g.ifrp));
  const float wfrp1 = one - wfrp;
  g.ifrm = static_cast<int>(std::log(one - c.lam) / xfrln);
  g.ifrm1 = g.ifrm - 1;
  const float wfrm = (powi(c.xfr, g.ifrm) - (one - c.lam)) /
                     (powi(c.xfr, g.ifrm) - powi(c.xfr, g.ifrm1));
  const float wfrm1 = one - wfrm;
  // 9. Interpolation weights.
  g.awg[0] = wthp * wfrp;
  g.awg[1] = wthp1 * wfrp;
  g.awg[2] = wthp * wfrp1;
  g.awg[3] = wthp1 * wfrp1;
  g.awg[4] = wthm * wfrm;
  g.awg[5] = wthm1 * wfrm;
  g.awg[6] = wthm * wfrm1;
  g.awg[7] = wthm1 * wfrm1;
  return g;
}

/// IF_m(IFR), m = 1..8, of section 7 (frequencies do not wrap; rows below 1 clamp to 0).
int if_map(const Geometry& g, int m, int ifr) {
  switch (m) {
    case 1: return ifr + g.ifrp;
    case 2: return ifr + g.ifrp1;
    case 3: return ifr + g.ifrm > 0 ? ifr + g.ifrm : 0;
    case 4: return ifr + g.ifrm1 > 0 ? ifr + g.ifrm1 : 0;
    case 5: return ifr - g.ifrp > 0 ? ifr - g.ifrp : 0;
    case 6: return ifr - g.ifrp1 > 0 ? ifr - g.ifrp1 : 0;
    case 7: return ifr - g.ifrm;
    default: return ifr - g.ifrm1;
  }
}

/// IT_n(ITH) - ITH before wrapping, n = 1..8.
void shifts(const Geometry& g, int out[8]) {
  out[0] = g.ithp;
  out[1] = g.ithp1;
  out[2] = g.ithm;
  out[3] = g.ithm1;
  out[4] = -g.ithp;
  out[5] = -g.ithp1;
  out[6] = -g.ithm;
  out[7] = -g.ithm1;
}

/// IT_n(ITH), 1-based, wrapped once as section 7 does (n <= 4 wrap down, n > 4 wrap up).
int it_map(const int sh[8], int n, int ith, int nth) {
  int v = ith + sh[n - 1];
  if (n <= 4) {
    if (v > nth) v -= nth;
  } else {
    if (v < 1) v += nth;
  }
  return v;
}

}  // namespace

bool build_snl1_tables(const Snl1Config& c, const float* sig, Snl1Tables& t) {
  t = Snl1Tables{};
  const int nth = c.nth, nspec = c.nspec();
  const Geometry g = geometry(c);
  t.nth = nth;
  t.nfr = c.nk;
  t.nspec = nspec;
  t.dal1 = g.dal1;
  t.dal2 = g.dal2;
  t.dal3 = g.dal3;
  for (int j = 0; j < 8; ++j) {
    t.awg[j] = g.awg[j];
    t.swg[j] = g.awg[j] * g.awg[j];
  }
  // 5. Range of the extended spectrum.
  t.nfrhgh = t.nfr + g.ifrp1 - g.ifrm1;
  t.nfrchg = t.nfr - g.ifrm1;
  t.nspecy = t.nfrhgh * nth;
  t.nspecx = t.nfrchg * nth;
  if (t.nfrchg <= 0 || t.nfrhgh < t.nfr) return false;

  // 7. Spectral addresses, stored minus one.
  int sh[8];
  shifts(g, sh);
  auto addr = [&](int n, int m, int ith, int ifr) {
    return it_map(sh, n, ith, nth) + (if_map(g, m, ifr) - 1) * nth - 1;
  };
  t.ipim.assign(16 * static_cast<size_t>(t.nspecx), 0);
  t.ic.assign(16 * static_cast<size_t>(nspec), 0);
  for (int isp = 0; isp < t.nspecx; ++isp) {
    const int ifr = 1 + isp / nth, ith = 1 + isp % nth;
    for (int j = 0; j < 16; ++j)
      t.ipim[static_cast<size_t>(j) * t.nspecx + isp] = addr(kPmMap[j][0], kPmMap[j][1], ith, ifr);
  }
  for (int isp = 0; isp < nspec; ++isp) {
    const int ifr = 1 + isp / nth, ith = 1 + isp % nth;
    for (int j = 0; j < 16; ++j)
      t.ic[static_cast<size_t>(j) * nspec + isp] = addr(kIcMap[j][0], kIcMap[j][1], ith, ifr);
  }

  // 8. AF11 = (f)**11 per frequency row; above NK the frequency grows by XFR per row.
  constexpr float kPi = static_cast<float>(3.141592653589793);
  constexpr float kTpiInv = 1.0f / (2.0f * kPi);
  t.af11.assign(static_cast<size_t>(t.nspecx), 0.0f);
  for (int ifr = 0; ifr < t.nfr; ++ifr) {
    const float v = pow11(sig[ifr] * kTpiInv);
    for (int ith = 0; ith < nth; ++ith) t.af11[ith + ifr * nth] = v;
  }
  float fr = sig[t.nfr - 1] * kTpiInv;
  for (int ifr = t.nfr; ifr < t.nfrchg; ++ifr) {
    fr = fr * c.xfr;
    const float v = pow11(fr);
    for (int ith = 0; ith < nth; ++ith) t.af11[ith + ifr * nth] = v;
  }
  derive_rowshift(c, t);
  return true;
}

bool build_snl1_weights_f64(const Snl1Config& c, const float* sig, const Snl1Tables& t,
                            Snl1WeightsF64& w) {
  const double one = 1.0, lam = c.lam, dth = c.dth, xfr = c.xfr;
  auto powi_d = [](double x, int n) {
    unsigned m = n < 0 ? static_cast<unsigned>(-n) : static_cast<unsigned>(n);
    double y = (m & 1u) ? x : 1.0;
    while ((m >>= 1u) != 0u) {
      x = x * x;
      if (m & 1u) y = y * x;
    }
    return n < 0 ? 1.0 / y : y;
  };
  auto pow11_d = [](double x) {
    const double x2 = x * x, x3 = x2 * x, x5 = x2 * x3, x6 = x3 * x3;
    return x5 * x6;
  };
  const double lamm2_b = one - lam, lamp2_b = one + lam;
  const double lamm2 = lamm2_b * lamm2_b, lamp2 = lamp2_b * lamp2_b;
  const double delth3 = std::acos((lamm2 * lamm2 + 4.0 - lamp2 * lamp2) / (4.0 * lamm2));
  const double delth4 = std::asin(-std::sin(delth3) * lamm2 / lamp2);
  const double p2 = lamp2_b * lamp2_b, m2 = lamm2_b * lamm2_b;
  w.dal1 = one / (p2 * p2);
  w.dal2 = one / (m2 * m2);
  w.dal3 = 2.0 * w.dal1 * w.dal2;
  const double cthp = std::fabs(delth4 / dth);
  const int ithp = static_cast<int>(cthp);
  const double wthp = cthp - ithp, wthp1 = one - wthp;
  const double cthm = std::fabs(delth3 / dth);
  const int ithm = static_cast<int>(cthm);
  const double wthm = cthm - ithm, wthm1 = one - wthm;
  const double xfrln = std::log(xfr);
  const int ifrp = static_cast<int>(std::log(one + lam) / xfrln), ifrp1 = ifrp + 1;
  const double wfrp = (one + lam - powi_d(xfr, ifrp)) / (powi_d(xfr, ifrp1) - powi_d(xfr, ifrp));
  const double wfrp1 = one - wfrp;
  const int ifrm = static_cast<int>(std::log(one - lam) / xfrln), ifrm1 = ifrm - 1;
  const double wfrm = (powi_d(xfr, ifrm) - (one - lam)) / (powi_d(xfr, ifrm) - powi_d(xfr, ifrm1));
  const double wfrm1 = one - wfrm;
  const Geometry gf = geometry(c);
  if (ithp != gf.ithp || ithm != gf.ithm || ifrp != gf.ifrp || ifrm != gf.ifrm) return false;
  w.awg[0] = wthp * wfrp;
  w.awg[1] = wthp1 * wfrp;
  w.awg[2] = wthp * wfrp1;
  w.awg[3] = wthp1 * wfrp1;
  w.awg[4] = wthm * wfrm;
  w.awg[5] = wthm1 * wfrm;
  w.awg[6] = wthm * wfrm1;
  w.awg[7] = wthm1 * wfrm1;
  for (int j = 0; j < 8; ++j) w.swg[j] = w.awg[j] * w.awg[j];
  const double tpiinv = 1.0 / (2.0 * 3.141592653589793);
  w.af11_row.assign(static_cast<size_t>(t.nfrchg), 0.0);
  for (int ifr = 0; ifr < t.nfr && ifr < t.nfrchg; ++ifr)
    w.af11_row[ifr] = pow11_d(static_cast<double>(sig[ifr]) * tpiinv);
  double fr = static_cast<double>(sig[t.nfr - 1]) * tpiinv;
  for (int ifr = t.nfr; ifr < t.nfrchg; ++ifr) {
    fr = fr * xfr;
    w.af11_row[ifr] = pow11_d(fr);
  }
  return true;
}

void derive_rowshift(const Snl1Config& c, Snl1Tables& t) {
  const int nth = c.nth;
  const Geometry g = geometry(c);
  t.rowshift = false;
  shifts(g, t.shift);
  t.ifrp = g.ifrp;
  t.ifrm = g.ifrm;
  t.ifrow.assign(8 * static_cast<size_t>(t.nfrchg), 0);
  for (int m = 1; m <= 8; ++m)
    for (int ifr = 1; ifr <= t.nfrchg; ++ifr)
      t.ifrow[static_cast<size_t>(m - 1) * t.nfrchg + (ifr - 1)] = if_map(g, m, ifr);
  // The wrapped column of a shift is only a single wrap when |shift| < NTH.
  for (int n = 0; n < 8; ++n)
    if (t.shift[n] >= nth || t.shift[n] <= -nth) return;
  // The row-shift form must give every stored entry (entry + NTH == row * NTH + column).
  auto same = [&](int stored, int n, int m, int isp) {
    const int ith0 = isp % nth, ifr0 = isp / nth;
    int col = ith0 + t.shift[n - 1];
    col = col < 0 ? col + nth : (col >= nth ? col - nth : col);
    const int row = t.ifrow[static_cast<size_t>(m - 1) * t.nfrchg + ifr0];
    return stored + nth == row * nth + col;
  };
  for (int isp = 0; isp < t.nspecx; ++isp)
    for (int j = 0; j < 16; ++j)
      if (!same(t.ipim[static_cast<size_t>(j) * t.nspecx + isp], kPmMap[j][0], kPmMap[j][1], isp))
        return;
  for (int isp = 0; isp < t.nspec; ++isp)
    for (int j = 0; j < 16; ++j)
      if (!same(t.ic[static_cast<size_t>(j) * t.nspec + isp], kIcMap[j][0], kIcMap[j][1], isp))
        return;
  // The rows the form reads must exist: section 3 reads UE rows 0..NFRHGH, section 4 reads the
  // interaction arrays at rows 0..NFRCHG.
  for (int ifr0 = 0; ifr0 < t.nfrchg; ++ifr0)
    for (int j = 0; j < 16; ++j) {
      const int row = t.ifrow[static_cast<size_t>(kPmMap[j][1] - 1) * t.nfrchg + ifr0];
      if (row < 0 || row > t.nfrhgh) return;
    }
  for (int ifr0 = 0; ifr0 < t.nfr; ++ifr0)
    for (int j = 0; j < 16; ++j) {
      const int row = t.ifrow[static_cast<size_t>(kIcMap[j][1] - 1) * t.nfrchg + ifr0];
      if (row < 0 || row > t.nfrchg) return;
    }
  // AF11 constant along each row.
  t.af11_row.assign(static_cast<size_t>(t.nfrchg), 0.0f);
  for (int ifr0 = 0; ifr0 < t.nfrchg; ++ifr0) {
    const float v = t.af11[static_cast<size_t>(ifr0) * nth];
    for (int ith = 0; ith < nth; ++ith)
      if (t.af11[static_cast<size_t>(ifr0) * nth + ith] != v) return;
    t.af11_row[ifr0] = v;
  }
  t.rowshift = true;
}

}  // namespace wwb
