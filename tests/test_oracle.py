"""The CPU oracle of the DIA, pinned before anything is checked against it.

* Against the reference's frozen golden vector (Fortran INSNL1 tables and W3SNL1 answers,
  kokkos/tests/fixtures/snl1_nk25_nth24.bin, converted by tests/golden/make_golden.py). That
  vector was produced by a -O0 gfortran build, whose AF11 = x**11 is libgcc's binary chain;
  the oracle's ``o0_chain`` option reproduces it (the reference documents the two chains in
  docs/log/2026-10-14-snl1-bitwise-af11.md).
* Against the reference's own C++ (snl1_tables.cpp, snl1_dia.cpp, snl1_shim.cpp) compiled
  unmodified into oracle/_ref/, where that build exists.
"""

import numpy as np
import pytest

from conftest import assert_bitexact


def test_tables_match_golden(oracle, golden):
    t = oracle.insnl1(golden["cfg"], golden["sig"], o0_chain=True)
    for key in ("scal", "ipim", "ic"):
        assert np.array_equal(t[key], golden[key]), key
    assert_bitexact(t["wts"], golden["wts"], "DAL/AWG/SWG")
    assert_bitexact(t["af11"], golden["af11"], "AF11 (-O0 chain)")


def test_af11_chains_differ_only_in_af11(oracle, golden):
    t3 = oracle.insnl1(golden["cfg"], golden["sig"], o0_chain=False)
    t0 = oracle.insnl1(golden["cfg"], golden["sig"], o0_chain=True)
    for key in ("scal", "wts", "ipim", "ic"):
        assert np.array_equal(t3[key], t0[key])
    # the two chains agree to a ULP or two, and differ in the last bit on many rows
    rel = np.abs(t3["af11"].astype(np.float64) / t0["af11"] - 1.0)
    assert rel.max() < 5e-7
    assert np.any(t3["af11"] != t0["af11"])


def test_w3snl1_matches_golden_bitexact(oracle, golden):
    s, d = oracle.w3snl1(golden["cfg"], golden["sig"], golden["a"], golden["cg"],
                         golden["kdmean"], o0_chain=True)
    assert_bitexact(s, golden["s"], "S vs Fortran")
    assert_bitexact(d, golden["d"], "D vs Fortran")


def test_golden_exercises_shallow_water(golden):
    # point 2 (10 m) has kdmean 1.73: CONS differs from SNLC1 there, so expf's bits matter
    assert golden["kdmean"].min() < 2.0 and golden["kdmean"].max() > 100.0


def test_f64_dia_close_to_f32(oracle, golden):
    s32, d32 = oracle.w3snl1(golden["cfg"], golden["sig"], golden["a"], golden["cg"],
                             golden["kdmean"])
    s64, d64 = oracle.w3snl1_f64(golden["cfg"], golden["sig"], golden["a"], golden["cg"],
                                 golden["kdmean"])
    scale = np.abs(s64).max(axis=1, keepdims=True)
    assert np.max(np.abs(s32 - s64) / scale) < 1e-5
    dscale = np.abs(d64).max(axis=1, keepdims=True)
    assert np.max(np.abs(d32 - d64) / dscale) < 1e-5


from oracle import oracle as _oracle  # noqa: E402

ref_missing = pytest.mark.skipif(not _oracle.ref_available(),
                                 reason="oracle/_ref not built (no reference checkout here)")


@ref_missing
def test_reference_build_tables_equal_oracle(oracle, golden, synth):
    for cfg, sig in ((golden["cfg"], golden["sig"]), synth.dia_config()):
        r = oracle.ref_tables(cfg, sig)
        t = oracle.insnl1(cfg, sig)
        for key in ("scal", "ipim", "ic"):
            assert np.array_equal(r[key], t[key]), key
        assert_bitexact(r["wts"], t["wts"], "weights")
        assert_bitexact(r["af11"], t["af11"], "AF11")


@ref_missing
@pytest.mark.parametrize("depth_range", [None, (5.0, 4000.0), (1.0, 20.0)])
def test_reference_build_w3snl1_equals_oracle(oracle, synth, depth_range):
    cfg, sig = synth.dia_config()
    g = synth.sea_states(200, seed=11, depth_range=depth_range, bimodal=0.2)
    ref = oracle.RefSnl1(cfg, sig, igrid=7)
    s_ref, d_ref = ref(g["a"], g["cg"], g["kdmean"])
    s, d = oracle.w3snl1(cfg, sig, g["a"], g["cg"], g["kdmean"])
    assert_bitexact(s, s_ref, "S")
    assert_bitexact(d, d_ref, "D")


@ref_missing
def test_reference_build_on_golden_inputs(oracle, golden):
    ref = oracle.RefSnl1(golden["cfg"], golden["sig"], igrid=8)
    s_ref, d_ref = ref(golden["a"], golden["cg"], golden["kdmean"])
    s, d = oracle.w3snl1(golden["cfg"], golden["sig"], golden["a"], golden["cg"],
                         golden["kdmean"])
    assert_bitexact(s, s_ref, "S")
    assert_bitexact(d, d_ref, "D")
