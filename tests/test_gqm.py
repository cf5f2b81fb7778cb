"""The GQM table builders (ww_snl1_gqm_couple on the device, ww_snl1_gqm_gauleg and
ww_snl1_gqm_f1f1f1 on the host) bit for bit against the reference's own C++
(kokkos/src/ww_kokkos/snl1_couple.hpp, snl1_gauleg.hpp, snl1_f1f1f1.hpp, compiled into oracle/_ref
and reached through oracle/ref_driver.cpp's ref_gqm_*), including COUPLE's degenerate terms and
every F1F1F1 layout with matching and mismatching NF1."""

import ctypes

import numpy as np
import pytest

from conftest import assert_bitexact, cuda_available
from oracle import oracle as _oracle

P, I = ctypes.c_void_p, ctypes.c_int
needs_ref = pytest.mark.skipif(not _oracle.ref_available(), reason="oracle/_ref not built")


def _lib(pkg):
    L = pkg.lib()
    L.ww_snl1_gqm_couple.argtypes = [I, P, P, P]
    L.ww_snl1_gqm_gauleg.argtypes = [I, P, P]
    L.ww_snl1_gqm_f1f1f1.argtypes = [P, I, P]
    for n in ("couple", "gauleg", "f1f1f1"):
        getattr(L, "ww_snl1_gqm_" + n).restype = I
    return L


def _ref():
    R = _oracle.ref_lib()
    R.ref_gqm_couple.argtypes = [I, P, P, P]
    R.ref_gqm_gauleg.argtypes = [I, P, P]
    R.ref_gqm_f1f1f1.argtypes = [P, I, P]
    return R


def p(x):
    return x.ctypes.data


@needs_ref
@pytest.mark.parametrize("npoin", [1, 2, 3, 6, 7, 10, 19, 40, 64])
def test_gauleg_equals_reference(pkg, npoin):
    L, R = _lib(pkg), _ref()
    w_r, x_r = np.full(npoin, 5.0), np.full(npoin, 5.0)
    R.ref_gqm_gauleg(npoin, p(w_r), p(x_r))
    w, x = np.full(npoin, 5.0), np.full(npoin, 5.0)
    assert L.ww_snl1_gqm_gauleg(npoin, p(w), p(x)) == 0
    assert_bitexact(w, w_r, f"W_LEG npoin {npoin}")
    assert_bitexact(x, x_r, f"X_LEG npoin {npoin}")
    assert abs(w.sum() - 2.0) < 1e-12  # the rule integrates 1 over [-1, 1]


@needs_ref
@pytest.mark.parametrize("iq_om1,nf1", [(1, 14), (1, 10), (2, 26), (2, 30), (3, 11), (3, 5),
                                        (4, 40), (4, 20), (5, 20), (5, 33), (6, 20), (6, 7),
                                        (7, 20), (7, 19), (0, 12), (8, 12)])
def test_f1f1f1_equals_reference(pkg, iq_om1, nf1):
    L, R = _lib(pkg), _ref()
    n_r, n = ctypes.c_int(nf1), ctypes.c_int(nf1)
    t_r, t = np.full(64, 7.0), np.full(64, 7.0)
    d_r = R.ref_gqm_f1f1f1(ctypes.byref(n_r), iq_om1, p(t_r))
    d = L.ww_snl1_gqm_f1f1f1(ctypes.byref(n), iq_om1, p(t))
    assert d == d_r and n.value == n_r.value
    assert_bitexact(t, t_r, f"F1SF layout {iq_om1} nf1 {nf1}")


def _quadruplets(n, seed):
    """Resonant-looking and random wavenumber quadruplets, with the degenerate cases COUPLE
    warns about: k3 = k1 (term 1-3 is 0/0) and k4 with |k1 - k4| = (sqrt k1 - sqrt k4)^2."""
    rng = np.random.default_rng(seed)
    k = rng.uniform(-0.5, 0.5, (n, 8))
    k[: n // 8, 4:6] = k[: n // 8, 0:2]           # k3 = k1
    k[n // 8: n // 4, 6:8] = k[n // 8: n // 4, 0:2]  # k4 = k1
    # k1 + k2 = k3 + k4 for a quarter of them (the resonance the quadrature samples)
    q = slice(n // 4, n // 2)
    k[q, 6:8] = k[q, 0:2] + k[q, 2:4] - k[q, 4:6]
    return np.ascontiguousarray(k)


@needs_ref
@pytest.mark.gpu
def test_couple_equals_reference(pkg):
    if not cuda_available():
        pytest.skip("needs a CUDA device")
    L, R = _lib(pkg), _ref()
    pkg.init()
    n = 100_003
    k = _quadruplets(n, 3)
    c_r, d_r = np.zeros(n), np.zeros(n, np.int32)
    R.ref_gqm_couple(n, p(k), p(c_r), p(d_r))
    c, d = np.zeros(n), np.full(n, -1, np.int32)
    assert L.ww_snl1_gqm_couple(n, p(k), p(c), p(d)) == 0
    assert np.array_equal(d, d_r)
    assert np.count_nonzero(d_r) > n // 8  # the planted degenerate terms are hit
    assert_bitexact(c, c_r, "COUPLE")
