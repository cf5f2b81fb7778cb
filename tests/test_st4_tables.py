"""INSIN4 on the device (ww_st4_tables, and ww_st4_commit under WW_KOKKOS_ST4_TABLES=1) bit for
bit against the reference's own host C++ INSIN4 / TABU_STRESS / TABU_TAUHF / TABU_TAUHF2
(kokkos/src/ww_kokkos/st4_insin4.cpp, st4_tabu_*.cpp, compiled into oracle/_ref and run through
oracle/ref_driver.cpp's ref_st4_tables): every entry of every table, and the DEL* scalars, on the
synthetic ST4 grids of every branch INSIN4 takes."""

import ctypes
import os
import time

import numpy as np
import pytest

from conftest import assert_bitexact, cuda_available

P, I = ctypes.c_void_p, ctypes.c_int
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


def _p(x):
    return None if x is None else x.ctypes.data


def _setup(synth, variant):
    st = synth.st4_setup(variant=variant if variant in ("default", "analytic", "romero")
                         else "default")
    R, r = st["R"], st["rpar"]
    if variant == "bck":  # the bandwidth-integrated breaking: IKTAB, DCKI, QBI built
        r[R["SSDSBCK"]] = 0.185
        r[R["SSDSBINT"]] = 0.3
        r[R["SSDSHCK"]] = 1.5
        r[R["SSDSABK"]] = 1.5
        r[R["SSDSPBK"]] = 4.0
    if variant == "plain":  # SSDSDTH >= 180 and SSDSC(3) >= 0: the fills without loops
        r[R["SSDSDTH"]] = 180.0
        r[R["SSDSC"] + 2] = 0.0
        r[R["TTAUWSHELTER"]] = 0.0  # TABU_TAUHF's own TAUHFT
    if variant == "odd":  # NTH odd, MK > NK, MTH > NTH, MSPEC > NSPEC, no cumulative band gap
        st = synth.st4_setup(nk=30, nth=25, xfr=1.1, f1=0.04)
        r, R = st["rpar"], st["R"]
        st["ipar"][3] = 32
        st["ipar"][4] = 27
        st["ipar"][5] = 32 * 27
        for key in ("sig", "dsip"):
            st[key] = np.concatenate([st[key], np.full(2, st[key][-1], np.float32)])
        st["th"] = np.concatenate([st["th"], np.zeros(2, np.float32)])
        nsp, nth = 30 * 25, 25
        ec = st["ecos"]
        st["ecos"] = np.concatenate([ec[:nsp], np.zeros(32 * 27 - nsp, np.float32), ec[nsp:],
                                     np.zeros(2, np.float32)])
        r[R["SSDSBRF1"]] = 0.0
    return st


def _device_tables(pkg, st, fltabs=1):
    L = pkg.lib()
    pkg.init()
    L.ww_st4_tables.argtypes = [P, I, P, I, P, P, P, P, I] + [P] * 10
    L.ww_st4_tables.restype = I
    ipar = st["ipar"]
    nk, nth, nspec, mk, mth, mspec = (int(v) for v in ipar[:6])
    nsat = 2 * (mth // 2 - 1) + 1
    R, r = st["R"], st["rpar"]
    tabs = fltabs and float(r[R["SINTAILPAR"]]) > 0.5
    tabs2 = tabs and float(r[R["TTAUWSHELTER"]]) > 0
    t = {"satweights": np.full(nsat * mth, 7.0, np.float32),
         "satindices": np.full(nsat * mth, 7, np.int32),
         "iktab": np.full(mk * 2000, 7, np.int32),
         "dcki": np.full(2000 * 1300, 7.0, np.float32),
         "qbi": np.full(2000 * 1300, 7.0, np.float32),
         "cumulw": np.full(mspec * mspec, 7.0, np.float32),
         "taut": np.full(201 * 201, 7.0, np.float32) if tabs else None,
         "tauhft": np.full(101 * 201, 7.0, np.float32) if tabs else None,
         "tauhft2": np.full(101 * 201 * 51, 7.0, np.float32) if tabs2 else None}
    dl = np.zeros(5, np.float32)
    t0 = time.perf_counter()
    rc = L.ww_st4_tables(_p(r), len(r), _p(ipar), len(ipar), _p(st["sig"]), _p(st["dsip"]),
                         _p(st["th"]), _p(st["ecos"]), fltabs, _p(t["satweights"]),
                         _p(t["satindices"]), _p(t["iktab"]), _p(t["dcki"]), _p(t["qbi"]),
                         _p(t["cumulw"]), _p(t["taut"]), _p(t["tauhft"]), _p(t["tauhft2"]),
                         _p(dl))
    t["seconds"] = time.perf_counter() - t0
    assert rc == 0, rc
    t["del"] = dl
    return t


def _compare(t, ref, what):
    for k in ("satweights", "satindices", "iktab", "dcki", "qbi", "cumulw", "taut", "tauhft",
              "tauhft2"):
        if ref.get(k) is None:
            assert t[k] is None, k
            continue
        assert_bitexact(t[k], ref[k], f"{what}: {k.upper()}")
    R = ref["R"]
    for j, name in enumerate(("DELUST", "DELALP", "DELTAUW", "DELU", "DELTAIL")):
        assert_bitexact(t["del"][j:j + 1], ref["rpar"][R[name]:R[name] + 1], f"{what}: {name}")


@pytest.mark.parametrize("variant", ["default", "analytic", "romero", "plain", "odd", "bck"])
def test_insin4_device_equals_reference(pkg, oracle, synth, variant):
    st = _setup(synth, variant)
    t0 = time.perf_counter()
    ref = oracle.st4_tables(st)
    cpu = time.perf_counter() - t0
    ref["R"] = st["R"]
    t = _device_tables(pkg, st)
    _compare(t, ref, variant)
    print(f"INSIN4 {variant}: device {t['seconds']:.3f} s, reference host C++ {cpu:.3f} s")


def test_commit_rebuilds_tables_on_the_device(pkg, oracle, synth, capfd):
    """WW_KOKKOS_ST4_TABLES=1: ww_st4_commit rebuilds the registered tables on the device and
    reports how many values differ: none when the registration is the reference's INSIN4 output,
    and every planted change otherwise (the rebuilt tables replace the planted ones)."""
    st = synth.st4_setup(variant="default")
    t = oracle.st4_tables(st)
    L = pkg.lib()
    pkg.init()
    old = os.environ.get("WW_KOKKOS_ST4_TABLES")
    os.environ["WW_KOKKOS_ST4_TABLES"] = "1"
    try:
        def reg(tt, igrid):
            return oracle.register_st4(lambda *a: L.ww_st4_init(igrid, *a),
                                       lambda *a: L.ww_st4_set_real(igrid, *a),
                                       lambda *a: L.ww_st4_set_int(igrid, *a),
                                       lambda: L.ww_st4_commit(igrid), st, tt)
        capfd.readouterr()
        assert reg(t, 231) == 0
        err = capfd.readouterr().err
        assert "ST4 tables rebuilt on the device: 0 values differ" in err, err
        planted = dict(t)
        planted["cumulw"] = t["cumulw"].copy()
        planted["cumulw"][:5] += 1.0
        planted["taut"] = t["taut"].copy()
        planted["taut"][300:303] *= 2.0  # J = 1: TAUT(I,0) is 0
        assert reg(planted, 232) == 0
        err = capfd.readouterr().err
        assert "ST4 tables rebuilt on the device: 8 values differ" in err, err
    finally:
        if old is None:
            del os.environ["WW_KOKKOS_ST4_TABLES"]
        else:
            os.environ["WW_KOKKOS_ST4_TABLES"] = old
