"""ST4 (W3SIN4, W3SDS4, W3SPR4) and W3SRCE: the kernels' source compiled for the host
(tests/hemu.cpp) against the reference's own build, bit for bit.

The reference is its C++ (oracle/_ref), built with the five libmvec loops of ST4 bound to scalar
glibc powf/expf per lane (libref_ww3_scalar.so), which is what any implementation without
libmvec computes; tables from the reference's own INSIN4/TABU_*. Three ST4 configurations
cover the saturation breaking with the cumulative term and tabulated stress (default), the
analytic tail with the Newton friction velocity (analytic) and Romero's breaking with its
libmvec loops (romero). The same comparison runs on the GPU in test_st4_gpu.py.
"""

import numpy as np
import pytest

from conftest import assert_bitexact
import st4_common as sc

VARIANTS = ["default", "analytic", "romero"]


@pytest.fixture(scope="module")
def hemu(tmp_path_factory):
    return sc.build_hemu(tmp_path_factory.mktemp("hemu"))


@pytest.fixture(scope="module")
def tables(oracle, synth):
    if not oracle.ref_available():
        pytest.skip("reference build absent")
    out = {}
    for v in VARIANTS:
        st = synth.st4_setup(variant=v)
        out[v] = (st, oracle.st4_tables(st))
    return out


@pytest.mark.parametrize("variant", VARIANTS)
def test_st4_terms_bitexact(oracle, synth, hemu, tables, variant):
    st, t = tables[variant]
    ref = oracle.RefSt4(st, t, igrid=11 + VARIANTS.index(variant), scalar_mvec=True)
    sc.setup_hemu(hemu, oracle, st, t)
    x = sc.point_inputs(synth.srce_points(48, seed=3))
    r = sc.run_all(sc.ref_backend(ref.L, ref.igrid), x)
    h = sc.run_all(sc.hemu_backend(hemu), x, llws=r["sin4"]["llws"])
    for term in ("sds4", "sin4", "spr4"):
        for k, v in r[term].items():
            if k == "llws":
                assert np.array_equal(v, h[term][k]), f"{term} {k}"
            else:
                assert_bitexact(h[term][k], v, f"{variant} {term} {k}")


@pytest.mark.parametrize("variant,ln1,seed,it", [("default", 0, 0, 1), ("analytic", 1, 1, 1),
                                                 ("romero", 0, 0, 0)])
def test_srce_batch_bitexact(oracle, synth, hemu, tables, variant, ln1, seed, it):
    st, t = tables[variant]
    sr = synth.srce_setup(st, ln1=ln1, seed=seed)
    dia = synth.dia_config()
    ref = oracle.RefSt4(st, t, igrid=21 + VARIANTS.index(variant), srce=sr, dia=dia,
                        scalar_mvec=True)
    sc.setup_hemu(hemu, oracle, st, t, srce=sr, dia=dia)
    pts = synth.srce_points(24, seed=11)
    r = sc.ref_backend(ref.L, ref.igrid).srce_batch(pts, it=it)
    assert ref.L.ww_srce_last_error() == 0
    h = sc.hemu_backend(hemu).srce_batch(pts, it=it)
    for k in ("spec", "psc", "whitecap", "taubbl", "tauice"):
        assert_bitexact(h[k], r[k], f"{variant} srce {k}")
    assert np.array_equal(h["shave"], r["shave"])


def _ulp(x, y):
    """Per-element distance in units in the last place between two float32 arrays."""
    def ordered(a):
        i = np.ascontiguousarray(a, np.float32).view(np.int32).astype(np.int64)
        return np.where(i >= 0, i, np.int64(-(2 ** 31)) - i)
    return np.abs(ordered(x) - ordered(y))


@pytest.mark.parametrize("variant", VARIANTS)
def test_max_ulp_against_libmvec_reference(oracle, synth, hemu, tables, variant, capsys):
    """The reference as built against this host's libmvec (4-lane SVML-style powf/expf) differs
    from any scalar-libm implementation at the libmvec sites of W3SDS4 / W3SIN4. The kernels
    follow the scalar binding (bit-exact above); this reports how far the as-built reference
    is, and bounds it."""
    st, t = tables[variant]
    ref = oracle.RefSt4(st, t, igrid=31 + VARIANTS.index(variant), scalar_mvec=False)
    sc.setup_hemu(hemu, oracle, st, t)
    x = sc.point_inputs(synth.srce_points(48, seed=3))
    r = sc.run_all(sc.ref_backend(ref.L, ref.igrid), x)
    h = sc.run_all(sc.hemu_backend(hemu), x, llws=r["sin4"]["llws"])
    lines = []
    for term in ("sds4", "sin4", "spr4"):
        for k, v in r[term].items():
            if k == "llws":
                continue
            u = _ulp(h[term][k], v)
            rel = np.abs(h[term][k].astype(np.float64) - v) / np.maximum(np.abs(v), 1e-30)
            lines.append(f"{variant:8s} {term} {k:10s} identical {np.mean(u == 0):7.2%} "
                         f"max ulp {int(u.max()):8d} max rel {float(rel.max()):.2e}")
            assert np.isfinite(h[term][k]).all()
            assert float(rel[np.abs(v) > 1e-20].max(initial=0.0)) < 1e-3, f"{term} {k}"
    with capsys.disabled():
        print("\n" + "\n".join(lines))
