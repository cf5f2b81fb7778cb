"""Seeded synthetic sea states for the DIA: JONSWAP spectra with cos^2s spreading.

The reference measures W3SNL1 on WW3 sea states (its frozen fixture and WW3 regtests); no such
data travels here, so these seeded spectra stand in, with the shapes and distributions of the
36x36 workload: frequencies geometric from 0.0373 Hz with ratio 1.1, 10-degree directions,
Hs ~ U(0.5, 8) m, fp ~ U(0.06, 0.2) Hz, gamma ~ U(1, 5), spreading cos^2s((th - thm)/2) with
s ~ U(2, 20) and a random mean direction thm. Intermediates are float64, outputs float32.

Action density and mean relative depth follow the reference's DIA benchmark generator
(ww3-gpu bench/dia/bench_dia.F90:81-107): A = E(sigma, theta) * Cg / sigma, with k and Cg from
the linear dispersion relation (Newton on sigma^2 = g k tanh(k d)) and
Cg = sigma / k / 2 * (1 + 2kd / sinh(min(2kd, 80))); KDMEAN = sum(E k d) / sum(E).
"""

import numpy as np

GRAV = 9.806  # ww3-gpu kokkos/src/ww_kokkos/st4_params.hpp:28
TPI_F32 = np.float32(2.0) * np.float32(np.pi)


def spectral_grid(nk=36, nth=36, f1=0.0373, xfr=1.1):
    """SIG(1:NK) (rad/s, float32, each a factor XFR above the last) and DTH = TPI / NTH."""
    xfr32 = np.float32(xfr)
    sig = np.empty(nk, np.float32)
    sig[0] = np.float32(TPI_F32 * np.float32(f1))
    for k in range(1, nk):
        sig[k] = np.float32(sig[k - 1] * xfr32)
    dth = np.float32(TPI_F32 / np.float32(nth))
    return sig, dth


def dia_config(nk=36, nth=36, xfr=1.1, lam=0.25, c_nl=2.78e7, kdconv=0.75, kdmin=0.5,
               cs1=5.5, cs2=0.833, cs3=-1.25, fachf=5.0):
    """ww_snl1_init's scalars for the DIA constants of the workload (SNLC1 = C / g^4,
    FACHFE = XFR^-FACHF)."""
    sig, dth = spectral_grid(nk, nth, xfr=xfr)
    cfg = {
        "nk": nk, "nth": nth, "xfr": float(np.float32(xfr)), "dth": float(dth),
        "lam": float(np.float32(lam)), "snlc1": float(np.float32(c_nl / GRAV ** 4)),
        "kdcon": float(np.float32(kdconv)), "kdmn": float(np.float32(kdmin)),
        "snls1": float(np.float32(cs1)), "snls2": float(np.float32(cs2)),
        "snls3": float(np.float32(cs3)),
        "fachfe": float(np.float32(np.float32(xfr) ** np.float32(-fachf))),
    }
    return cfg, sig


def wavenumber(sig, depth, iters=30):
    """k(sigma, d) from sigma^2 = g k tanh(k d), Newton from the deep-water value; float64.
    sig (nk,), depth (npts,) -> k (npts, nk)."""
    s = np.asarray(sig, np.float64)[None, :]
    d = np.asarray(depth, np.float64)[:, None]
    k = np.broadcast_to(s * s / GRAV, (d.shape[0], s.shape[1])).copy()
    for _ in range(iters):
        kd = np.minimum(k * d, 40.0)
        t = np.tanh(kd)
        f = GRAV * k * t - s * s
        fp = GRAV * t + GRAV * k * d / np.cosh(kd) ** 2
        k = k - f / fp
    return k


def sea_states(npts, seed=0, nk=36, nth=36, depth=4000.0, depth_range=None, bimodal=0.0):
    """npts seeded JONSWAP points: returns dict(a (npts, nspec), cg (npts, nk), kdmean (npts,),
    depth (npts,), hs (npts,)) with float32 spectra. ``depth_range=(lo, hi)`` draws depths
    log-uniformly instead of the fixed ``depth``; ``bimodal`` is the fraction of points that get
    an added swell system."""
    rng = np.random.default_rng(seed)
    cfg, sig = dia_config(nk, nth)
    dth = np.float64(cfg["dth"])
    s64 = sig.astype(np.float64)
    f = s64 / (2 * np.pi)
    th = np.arange(nth) * dth
    xfr = np.float64(cfg["xfr"])
    dsii = 0.5 * s64 * (xfr - 1.0 / xfr)  # band widths in sigma

    hs = rng.uniform(0.5, 8.0, npts)
    fp = rng.uniform(0.06, 0.2, npts)
    gam = rng.uniform(1.0, 5.0, npts)
    spr = rng.uniform(2.0, 20.0, npts)
    thm = rng.uniform(0.0, 2 * np.pi, npts)
    if depth_range is None:
        dep = np.full(npts, float(depth))
    else:
        lo, hi = depth_range
        dep = np.exp(rng.uniform(np.log(lo), np.log(hi), npts))
    swell = rng.uniform(0, 1, npts) < bimodal
    hs_sw = rng.uniform(0.5, 3.0, npts)
    fp_sw = rng.uniform(0.05, 0.09, npts)
    thm_sw = rng.uniform(0.0, 2 * np.pi, npts)

    def jonswap(fpk, gk):
        ff = f[None, :]
        fpp = fpk[:, None]
        sg = np.where(ff <= fpp, 0.07, 0.09)
        r = np.exp(-((ff - fpp) ** 2) / (2.0 * sg * sg * fpp * fpp))
        return ff ** -5 * np.exp(-1.25 * (fpp / ff) ** 4) * gk[:, None] ** r

    def spreading(tm, sk):
        x = np.cos(0.5 * (th[None, :] - tm[:, None])) ** 2
        dd = x ** sk[:, None]
        return dd / (dd.sum(axis=1, keepdims=True) * dth)

    def energy(hsk, fpk, gk, tm, sk):
        ef = jonswap(fpk, gk) / (2 * np.pi)  # density in sigma
        e = ef[:, :, None] * spreading(tm, sk)[:, None, :]  # (npts, nk, nth)
        m0 = (e * dsii[None, :, None]).sum(axis=(1, 2)) * dth
        return e * ((hsk / 4.0) ** 2 / m0)[:, None, None]

    e = energy(hs, fp, gam, thm, spr)
    if swell.any():
        idx = np.nonzero(swell)[0]
        e[idx] += energy(hs_sw[idx], fp_sw[idx], np.full(idx.size, 3.3), thm_sw[idx],
                         np.full(idx.size, 20.0))
    k = wavenumber(sig, dep)
    kd = k * dep[:, None]
    cg = 0.5 * s64[None, :] / k * (1.0 + 2.0 * kd / np.sinh(np.minimum(2.0 * kd, 80.0)))
    a = e * (cg / s64[None, :])[:, :, None]
    esum = e.sum(axis=2)
    kdmean = (esum * kd).sum(axis=1) / np.maximum(esum.sum(axis=1), np.finfo(np.float64).tiny)
    m0 = (e * dsii[None, :, None]).sum(axis=(1, 2)) * dth
    return {
        "a": a.reshape(npts, nk * nth).astype(np.float32),
        "cg": cg.astype(np.float32),
        "kdmean": kdmean.astype(np.float32),
        "depth": dep.astype(np.float32),
        "hs": (4.0 * np.sqrt(m0)).astype(np.float32),
    }


def sea_states_chunked(npts, seed=0, chunk=32768, out=None, **kw):
    """sea_states for large npts, chunk by chunk (chunk j seeded seed*1_000_003 + j), written
    into ``out`` = dict of preallocated arrays when given."""
    nk, nth = kw.get("nk", 36), kw.get("nth", 36)
    if out is None:
        out = {"a": np.empty((npts, nk * nth), np.float32), "cg": np.empty((npts, nk), np.float32),
               "kdmean": np.empty(npts, np.float32)}
    for j, p0 in enumerate(range(0, npts, chunk)):
        n = min(chunk, npts - p0)
        g = sea_states(n, seed=seed * 1_000_003 + j, **kw)
        for key in out:
            out[key][p0:p0 + n] = g[key]
    return out
