"""ST4 (ww_sds4, ww_sin4, ww_spr4) and W3SRCE (ww_srce_batch, ww_srce_batch_va, ww_srce) on the
GPU through the C ABI, bit for bit against the reference's own build.

The reference is its C++ (oracle/_ref, libref_ww3_scalar.so: the five libmvec loops of ST4 run
scalar glibc powf/expf per lane, the arithmetic a device without libmvec has); its tables come
from its own INSIN4/TABU_*, and both sides get the same registered arrays. The CPU tests
(test_st4_host.py) check the same kernels' source compiled for the host.
"""

import numpy as np
import pytest

from conftest import assert_bitexact, cuda_available
import st4_common as sc

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

VARIANTS = ["default", "analytic", "romero"]


@pytest.fixture(scope="module")
def tables(oracle, synth):
    out = {}
    for v in VARIANTS:
        st = synth.st4_setup(variant=v)
        out[v] = (st, oracle.st4_tables(st))
    return out


def gpu_setup(pkg, oracle, synth, st, t, igrid, srce=None):
    L = pkg.lib()
    pkg.init()
    rc = oracle.register_st4(lambda *a: L.ww_st4_init(igrid, *a),
                             lambda *a: L.ww_st4_set_real(igrid, *a),
                             lambda *a: L.ww_st4_set_int(igrid, *a),
                             lambda: L.ww_st4_commit(igrid), st, t)
    assert rc == 0, rc
    if srce is not None:
        cfg, sig = synth.dia_config()
        pkg.Snl1Grid(cfg, sig, igrid=igrid)
        rc = L.ww_srce_init(igrid, sc.p(srce["rpar"]), len(srce["rpar"]), sc.p(srce["ipar"]),
                            len(srce["ipar"]), sc.p(srce["sig"]), sc.p(srce["dden"]),
                            sc.p(srce["ecos"]), sc.p(srce["esin"]), sc.p(srce["mapwn"]))
        assert rc == 0, rc
    return L, sc.Backend(lambda name: (lambda *a: getattr(L, "ww_" + name)(igrid, *a)))


@pytest.mark.parametrize("variant", VARIANTS)
def test_st4_terms_bitexact(pkg, oracle, synth, tables, variant):
    st, t = tables[variant]
    ig = 200 + VARIANTS.index(variant)
    ref = oracle.RefSt4(st, t, igrid=ig, scalar_mvec=True)
    L, be = gpu_setup(pkg, oracle, synth, st, t, ig)
    x = sc.point_inputs(synth.srce_points(300, seed=4))
    r = sc.run_all(sc.ref_backend(ref.L, ig), x)
    g = sc.run_all(be, x, llws=r["sin4"]["llws"])
    assert L.ww_st4_last_error() == 0
    for term in ("sds4", "sin4", "spr4"):
        for k, v in r[term].items():
            if k == "llws":
                assert np.array_equal(v, g[term][k]), f"{term} {k}"
            else:
                assert_bitexact(g[term][k], v, f"{variant} {term} {k}")


@pytest.mark.parametrize("variant,ln1,seed,it,npts", [("default", 0, 0, 1, 9520),
                                                      ("analytic", 1, 1, 1, 500),
                                                      ("romero", 0, 0, 0, 500)])
def test_srce_batch_bitexact(pkg, oracle, synth, tables, variant, ln1, seed, it, npts):
    """ww_srce_batch; the default case is the full W3SRCE workload: 9520 points, 36x36, depths
    log-uniform in 10-4000 m, U10 in 3-25 m/s, DTG = 900 s with dynamic substeps."""
    st, t = tables[variant]
    ig = 210 + VARIANTS.index(variant)
    sr = synth.srce_setup(st, ln1=ln1, seed=seed)
    ref = oracle.RefSt4(st, t, igrid=ig, srce=sr, dia=synth.dia_config(), scalar_mvec=True)
    L, be = gpu_setup(pkg, oracle, synth, st, t, ig, srce=sr)
    pts = synth.srce_points(npts, seed=2026)
    r = sc.ref_backend(ref.L, ig).srce_batch(pts, it=it)
    assert ref.L.ww_srce_last_error() == 0
    g = be.srce_batch(pts, it=it)
    assert L.ww_srce_last_error() == 0
    for k in ("spec", "psc", "whitecap", "taubbl", "tauice"):
        assert_bitexact(g[k], r[k], f"{variant} srce {k}")
    assert np.array_equal(g["shave"], r["shave"])


def test_srce_bench_workload_bitexact(pkg, oracle, synth):
    """Exactly the inputs bench.py's W3SRCE line times: the analytic-tail ST4 configuration with
    this project's own ST4 tables (synth.st4_tables_own, registered on both sides), the default
    W3SRCE packets, 9520 points of seed 2026. The reference's C++ (scalar-libmvec build) and the
    GPU agree bit for bit through the host entry ww_srce_batch and the device entry
    ww_srce_batch_device the bench calls."""
    import torch

    st = synth.st4_setup(variant="analytic")
    t = synth.st4_tables_own(st)
    sr = synth.srce_setup(st)
    ig = 240
    ref = oracle.RefSt4(st, t, igrid=ig, srce=sr, dia=synth.dia_config(), scalar_mvec=True)
    L, be = gpu_setup(pkg, oracle, synth, st, t, ig, srce=sr)
    pts = synth.srce_points(9520, seed=2026)
    r = sc.ref_backend(ref.L, ig).srce_batch(pts, it=1)
    assert ref.L.ww_srce_last_error() == 0
    g = be.srce_batch(pts, it=1)
    assert L.ww_srce_last_error() == 0
    for k in ("spec", "psc", "whitecap", "taubbl", "tauice"):
        assert_bitexact(g[k], r[k], f"bench workload, host entry, {k}")
    assert np.array_equal(g["shave"], r["shave"])
    dv = {k: torch.from_numpy(np.ascontiguousarray(pts[k])).cuda()
          for k in ("spec", "wn1", "cg1", "pin", "psc", "whitecap", "taubbl", "tauice")}
    shave = torch.zeros(9520, dtype=torch.int32, device="cuda")
    L.ww_srce_batch_device(ig, 1, 0, 1, 1, 900.0, 9520,
                           *[dv[k].data_ptr() for k in ("spec", "wn1", "cg1", "pin", "psc",
                                                        "whitecap", "taubbl", "tauice")],
                           shave.data_ptr(), None)
    torch.cuda.synchronize()
    assert L.ww_srce_last_error() == 0
    for k in ("spec", "psc", "whitecap", "taubbl", "tauice"):
        assert_bitexact(dv[k].cpu().numpy(), r[k], f"bench workload, device entry, {k}")
    assert np.array_equal(shave.cpu().numpy(), r["shave"])


def test_srce_autotune_keeps_results_bitexact(pkg, oracle, synth, tables):
    """ww_srce_autotune times the W3SRCE kernel at every CTA count per SM on device copies of
    the caller's points (the host arrays stay as they were), keeps the fastest, and the
    batches after it still give the reference's bits."""
    st, t = tables["default"]
    ig = 225
    sr = synth.srce_setup(st)
    ref = oracle.RefSt4(st, t, igrid=ig, srce=sr, dia=synth.dia_config(), scalar_mvec=True)
    L, be = gpu_setup(pkg, oracle, synth, st, t, ig, srce=sr)
    pts = synth.srce_points(700, seed=2027)
    before = {k: np.array(v, copy=True) for k, v in pts.items()}
    c = pkg.srce_autotune(ig, pts)
    assert c >= 1
    for k in before:
        assert np.array_equal(pts[k], before[k]), k
    rep = pkg.autotune_report()
    key = next(x for x in rep if x.startswith("srce ctas/SM 36x36"))
    assert rep[key]["choice"] == c
    r = sc.ref_backend(ref.L, ig).srce_batch(pts, it=1)
    g = be.srce_batch(pts, it=1)
    assert L.ww_srce_last_error() == 0
    for k in ("spec", "psc", "whitecap", "taubbl", "tauice"):
        assert_bitexact(g[k], r[k], f"after autotune, {k}")
    assert np.array_equal(g["shave"], r["shave"])


def test_srce_batch_va_and_single_point(pkg, oracle, synth, tables):
    """The resident-VA batch writes the same spectra into the VA columns JSEA names, and the
    one-point entry ww_srce gives the batch's result for that point."""
    st, t = tables["default"]
    ig = 220
    sr = synth.srce_setup(st)
    L, be = gpu_setup(pkg, oracle, synth, st, t, ig, srce=sr)
    npts, nsealm, nspec = 64, 100, 1296
    pts = synth.srce_points(npts, seed=31)
    want = be.srce_batch(pts)
    rng = np.random.default_rng(5)
    jsea = np.sort(rng.choice(np.arange(1, nsealm + 1), npts, replace=False)).astype(np.int32)
    va = np.zeros((nsealm + 1, nspec), np.float32)
    va[jsea] = pts["spec"]
    rest = {k: pts[k].copy() for k in ("psc", "whitecap", "taubbl", "tauice")}
    shave = np.zeros(npts, np.int32)
    L.ww_srce_batch_va(ig, 1, 0, 1, 1, 900.0, sc.p(va), nspec, nsealm, npts, sc.p(jsea),
                       sc.p(pts["wn1"]), sc.p(pts["cg1"]), sc.p(pts["pin"]), sc.p(rest["psc"]),
                       sc.p(rest["whitecap"]), sc.p(rest["taubbl"]), sc.p(rest["tauice"]),
                       sc.p(shave))
    assert L.ww_srce_last_error() == 0
    assert L.ww_va_host_read(ig, sc.p(va), nspec, nsealm) == 0
    assert_bitexact(va[jsea], want["spec"], "VA columns")
    assert_bitexact(rest["psc"], want["psc"], "psc (VA)")
    # ww_srce on point 3
    k = 3
    spec = pts["spec"][k].copy()
    sc_ = [np.array([v], np.float32) for v in pts["psc"][k]]
    wc, tb, ti = pts["whitecap"][k].copy(), pts["taubbl"][k].copy(), pts["tauice"][k].copy()
    sh = np.zeros(1, np.int32)
    pin = pts["pin"][k]
    wn1k, cg1k = pts["wn1"][k].copy(), pts["cg1"][k].copy()  # kept alive across the call
    args = [sc.p(a) for a in sc_[:16]] + [sc.p(wc), sc.p(sc_[16]), sc.p(tb), sc.p(ti)] + \
        [sc.p(a) for a in sc_[17:22]] + [sc.p(sh)]
    L.ww_srce(ig, 1, 0, 1, 1, sc.p(spec), sc.p(wn1k), sc.p(cg1k),
              float(pin[0]), float(pin[1]), float(pin[2]), float(pin[3]), float(pin[4]), 900.0,
              float(pin[5]), float(pin[6]), *args)
    assert L.ww_srce_last_error() == 0
    assert_bitexact(spec, want["spec"][k], "ww_srce spec")
    assert_bitexact(np.concatenate(sc_), want["psc"][k], "ww_srce scalars")


def test_st4_and_srce_validation(pkg, oracle, synth, tables):
    L = pkg.lib()
    pkg.init()
    st, t = tables["default"]
    r = np.zeros(84, np.float32)
    i = np.zeros(9, np.int32)
    assert L.ww_st4_init(230, sc.p(r), 83, sc.p(i), 9) == pkg.ERR_BAD_SHAPE
    i2 = st["ipar"].copy()
    i2[8] = 1  # W3_FLX5
    assert L.ww_st4_init(230, sc.p(t["rpar"]), 84, sc.p(i2), 9) == 5
    assert L.ww_st4_init(230, sc.p(t["rpar"]), 84, sc.p(st["ipar"]), 9) == 0
    assert L.ww_st4_commit(230) == 6  # nothing registered
    lb, ext = np.array([1], np.int32), np.array([36], np.int32)
    assert L.ww_st4_set_real(230, 0, sc.p(st["sig"]), 1, sc.p(lb), sc.p(ext)) == 6  # SIG lb is 0
    sr = synth.srce_setup(st)
    assert L.ww_srce_init(231, sc.p(sr["rpar"]), 29, sc.p(sr["ipar"]), 12, sc.p(sr["sig"]),
                          sc.p(sr["dden"]), sc.p(sr["ecos"]), sc.p(sr["esin"]),
                          sc.p(sr["mapwn"])) == pkg.ERR_NOT_INITIALISED
    ip = sr["ipar"].copy()
    ip[7] = 0
    assert L.ww_srce_init(231, sc.p(sr["rpar"]), 29, sc.p(ip), 12, sc.p(sr["sig"]),
                          sc.p(sr["dden"]), sc.p(sr["ecos"]), sc.p(sr["esin"]),
                          sc.p(sr["mapwn"])) == 5
    spec = np.zeros(1296, np.float32)
    L.ww_srce_batch(232, 1, 0, 1, 1, 900.0, 1, sc.p(spec), None, None, None, None, None, None,
                    None, None)
    assert L.ww_srce_last_error() == pkg.ERR_NOT_INITIALISED
