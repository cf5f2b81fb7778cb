"""W3OUTG on the device (ww_outg_va, ww_outg_part) against the reference's own W3OUTG
(kokkos/src/ww_kokkos/iogo_w3outg.hpp through kokkos/src/fortran_iface/outg_shim.cpp, compiled
into oracle/_ref/libref_ww3_scalar.so, whose host path writes every field in place). Every field
the call sends back must equal the reference's bit for bit; every field it does not send back
must keep the caller's bits (the reference's device path copies back only what W3IOGO and
W3IORS read). Seeded grids with active, boundary and excluded sea points, calm points, shallow
and deep water, both MAXSS orders (OMPG), every branch of the space-time extremes, and the
partition fields of W3CPRT's table."""

import ctypes
from pathlib import Path

import numpy as np
import pytest

from conftest import assert_bitexact, cuda_available
from oracle import oracle as _oracle

P, I = ctypes.c_void_p, ctypes.c_int
SCALAR_REF = Path(_oracle.REF_PATH).parent / "libref_ww3_scalar.so"
needs_ref = pytest.mark.skipif(not SCALAR_REF.exists(), reason="oracle/_ref not built")

OK, NOT_INIT, BAD_SHAPE, UNSUPPORTED = 0, 1, 2, 5
# The (group, index) entries of FLOGRD (W3IOGO) and FLOGRR (W3IORS) that read each field of
# outg_c.hpp's WwOutgField order (outg_shim.cpp:94-150).
GRD = [[(2, 1)], [(2, 2)], [(2, 3)], [(2, 4)], [(2, 5)], [(2, 6), (2, 18)], [(2, 7)], [(2, 8)],
       [(2, 9)], [(2, 10)], [(8, 6)], [(8, 5)], [(2, 17)], [(2, 11)], [(2, 12)], [(2, 14)],
       [(2, 13)], [(2, 16)], [(2, 15)], [(7, 1)], [(7, 1)], [(7, 2)], [(7, 2)], [(6, 1)],
       [(6, 1)], [(6, 1)], [(6, 6)], [(6, 6)], [(6, 5)], [(6, 5)], [(8, 1)], [(8, 1)], [(8, 3)],
       [(8, 2)], [(8, 2)], [(8, 4)], [(6, 7)], [(6, 7)], [(6, 3)], [(5, 3)], [(3, 1)], [(3, 2)],
       [(3, 3)], [(3, 4)], [(3, 5)], [(6, 9)]]
GRR = {0: [(2, 1)], 1: [(2, 2)], 3: [(2, 4)], 4: [(2, 5)], 5: [(2, 6)], 6: [(2, 7)],
       21: [(7, 2)], 22: [(7, 2)], 26: [(6, 6)], 27: [(6, 6)], 28: [(6, 5)], 29: [(6, 5)],
       38: [(6, 3)]}
NAMES = ("HS WLM T02 T0M1 T01 FP0 THM THS THP0 HSIG QKK QP WBT STMAXE STMAXD HCMAXE HMAXE HCMAXD "
         "HMAXD ABA ABD UBA UBD SXX SYY SXY USSX USSY TUSX TUSY MSSX MSSY MSSD MSCX MSCY MSCD PRMS "
         "TPMS BHD CGE EF TH1M STH1M TH2M STH2M P2SMS").split()


def _bind(L):
    L.ww_outg_va.argtypes = [I, P, I, P, I, P, P, P, P, I, I] + [P] * 13 + [P, I]
    L.ww_outg_va.restype = I
    L.ww_outg_part.argtypes = [P, I, P, I] + [P] * 6 + [P, I]
    L.ww_outg_part.restype = I
    return L


def _ref():
    return _bind(_oracle._ref_variant(SCALAR_REF))


def _gpu_lib(pkg):
    if not cuda_available():
        pytest.skip("needs a CUDA device")
    L = pkg.lib()
    pkg.init()
    return _bind(L)


def _wanted(c):
    """The fields ww_outg_va sends back for case c (floutg, floutg2, oarst of its ipar)."""
    nog = 10
    ip = c["ipar"]
    floutg, floutg2, oarst = ip[9] != 0, ip[10] != 0, ip[11] != 0

    def lg(f, i, j):
        return f[(i - 1) + (j - 1) * nog] != 0

    def floloc(i, j):
        return (floutg and lg(c["flogrd"], i, j)) or (floutg2 and lg(c["flogr2"], i, j))

    out = []
    for k in range(46):
        w = any(floloc(i, j) for i, j in GRD[k])
        if oarst:
            w = w or any(lg(c["flogrr"], i, j) for i, j in GRR.get(k, []))
        out.append(w)
    return out


def call_outg(L, igrid, c, fields, va, ipar=None, nipar=25):
    ip = c["ipar"] if ipar is None else ipar
    ptrs = (ctypes.c_void_p * 46)(*[f.ctypes.data if f is not None else None for f in fields])
    a = [c[k].ctypes.data for k in ("cg", "wn", "dw", "sig", "dden", "dsii", "ecos", "esin",
                                    "ec2", "es2", "esc", "mapsf", "mapsta")]
    return L.ww_outg_va(igrid, ip.ctypes.data, nipar, c["rpar"].ctypes.data, 10,
                        c["flogrd"].ctypes.data, c["flogr2"].ctypes.data, c["flogrr"].ctypes.data,
                        va.ctypes.data, va.shape[1], va.shape[0] - 1, *a, ptrs, 46)


def call_part(L, c, fields, nipar=13):
    ptrs = (ctypes.c_void_p * 17)(*[f.ctypes.data for f in fields])
    return L.ww_outg_part(c["ipar"].ctypes.data, nipar, c["rpar"].ctypes.data, 2,
                          c["flogrd"].ctypes.data, c["flogr2"].ctypes.data,
                          c["mapsf"].ctypes.data, c["mapsta"].ctypes.data,
                          c["icprt"].ctypes.data, c["dtprt"].ctypes.data, ptrs, 17)


def _copy_fields(fields):
    return [None if f is None else np.array(f, copy=True) for f in fields]


CASES = [  # (name, synth.outg_case keywords)
    ("all-shrd-ste", dict(seed=1, ompg=0, ste=(1000.0, 1000.0, 3600.0))),
    ("all-ompg-time", dict(seed=2, ompg=1, ste=(0.0, 0.0, 3600.0))),
    ("some-space", dict(seed=3, ompg=0, ste=(1000.0, 1000.0, 0.0), select="some", floutg2=1,
                        oarst=1)),
    ("all-no-ste", dict(seed=4, ompg=0, ste=(0.0, 0.0, 0.0))),
    ("all-large", dict(nx=120, ny=80, seed=5, ompg=0, ste=(2000.0, 500.0, 1800.0), nk=36,
                       nth=36)),
    ("empty", dict(seed=6, nseal0=True)),
    ("e3df-outside", dict(seed=7, e3df=([0, 3, -2, 2, 5], [30, 33, 12, 20, 29]), p2=(-1, 4))),
]


@needs_ref
@pytest.mark.gpu
@pytest.mark.parametrize("name,kw", CASES, ids=[c[0] for c in CASES])
def test_outg_va_equals_reference(pkg, synth, name, kw):
    L = _gpu_lib(pkg)
    R = _ref()
    kw = dict(kw)
    nseal0 = kw.pop("nseal0", False)
    c = synth.outg_case(**kw)
    if nseal0:
        c["ipar"][2] = 0  # NSEAL = 0: only the whole-array assignments of section 1
    ig = 800 + [x[0] for x in CASES].index(name)
    f_ref = _copy_fields(c["fields"])
    va_ref = np.array(c["va"], copy=True)
    assert call_outg(R, ig, c, f_ref, va_ref) == OK
    f_gpu = _copy_fields(c["fields"])
    va_gpu = np.array(c["va"], copy=True)
    assert call_outg(L, ig, c, f_gpu, va_gpu) == OK
    want = _wanted(c)
    assert any(want)
    for k in range(46):
        if want[k]:
            assert_bitexact(f_gpu[k], f_ref[k], f"{name}: {NAMES[k]}")
        else:
            assert_bitexact(f_gpu[k], c["fields"][k], f"{name}: {NAMES[k]} not sent back")
    assert np.array_equal(va_gpu.view(np.uint32), c["va"].view(np.uint32))
    # A second call on the same resident VA (device state now current) gives the same bits.
    f_again = _copy_fields(c["fields"])
    assert call_outg(L, ig, c, f_again, va_gpu) == OK
    for k in range(46):
        assert_bitexact(f_again[k], f_gpu[k], f"{name}: {NAMES[k]}, second call")


@needs_ref
@pytest.mark.gpu
@pytest.mark.parametrize("seed,noswll,select", [(1, 3, "all"), (2, 0, "all"), (3, 5, "some")])
def test_outg_part_equals_reference(pkg, synth, seed, noswll, select):
    L = _gpu_lib(pkg)
    R = _ref()
    c = synth.outg_part_case(seed=seed, noswll=noswll, select=select)
    f_ref = _copy_fields(c["fields"])
    assert call_part(R, c, f_ref) == OK
    f_gpu = _copy_fields(c["fields"])
    assert call_part(L, c, f_gpu) == OK
    for k in range(17):
        if c["flogrd"][3 + k * 10]:
            assert_bitexact(f_gpu[k], f_ref[k], f"partition field {k}")
        else:
            assert_bitexact(f_gpu[k], c["fields"][k], f"partition field {k} not sent back")


# ------------------------------------------------------------ host checks (no device needed)
@needs_ref
def test_outg_statuses_match_reference(pkg, synth):
    """The packet and request checks run before any device work: each bad call returns the
    reference's status (the library is not initialised here, so a good call says so)."""
    L = _bind(pkg.lib())
    R = _ref()
    c = synth.outg_case(seed=7)
    va = np.array(c["va"], copy=True)
    f = _copy_fields(c["fields"])
    assert call_outg(L, 1, c, f, va, nipar=24) == BAD_SHAPE
    assert call_outg(R, 901, c, f, va, nipar=24) == BAD_SHAPE
    for i, j in ((6, 8), (6, 12), (8, 7), (8, 8), (8, 9), (2, 17)):
        c2 = dict(c)
        c2["flogrd"] = np.array(c["flogrd"], copy=True)
        c2["flogrd"][(i - 1) + (j - 1) * 10] = 1
        assert call_outg(L, 1, c2, f, va) == UNSUPPORTED
        assert call_outg(R, 902, c2, f, va) == UNSUPPORTED
    f_null = list(f)
    f_null[41] = None  # TH1M requested and not allocated
    assert call_outg(L, 1, c, f_null, va) == BAD_SHAPE
    assert call_outg(R, 903, c, f_null, va) == BAD_SHAPE
    bad = np.array(c["ipar"], copy=True)
    bad[2] = bad[6] + 1  # NSEAL > NFLD
    assert call_outg(L, 1, c, f, va, ipar=bad) == BAD_SHAPE
    assert call_outg(R, 904, c, f, va, ipar=bad) == BAD_SHAPE
    # the library's own check: a MAPSF cell outside the grid
    c3 = dict(c)
    c3["mapsf"] = np.array(c["mapsf"], copy=True)
    c3["mapsf"][0] = int(c["ipar"][4]) + 1
    assert call_outg(L, 1, c3, f, va) == BAD_SHAPE
    if not cuda_available():
        assert call_outg(L, 1, c, f, va) == NOT_INIT
    p = synth.outg_part_case(seed=8)
    fp = _copy_fields(p["fields"])
    assert call_part(L, p, fp, nipar=12) == BAD_SHAPE
    assert call_part(R, p, fp, nipar=12) == BAD_SHAPE
    p2 = dict(p)
    p2["icprt"] = np.array(p["icprt"], copy=True)
    ns, ny = p["nsea"], int(p["ipar"][3])
    sea = np.nonzero(p["mapsta"][(p["mapsf"][:ns] - 1) * ny + p["mapsf"][ns:2 * ns] - 1] > 0)[0]
    nicp = int(p["ipar"][6])
    p2["icprt"][sea[0]] = 3
    p2["icprt"][nicp + sea[0]] = int(p["ipar"][7])  # the last column: two past the end
    assert call_part(L, p2, fp) == BAD_SHAPE
    if not cuda_available():
        assert call_part(L, p, fp) == NOT_INIT


def test_outg_case_shapes(synth):
    c = synth.outg_case(seed=9)
    nsealm = c["nsealm"]
    assert c["va"].shape == (nsealm + 1, 30 * 24)
    assert c["cg"].shape == (c["nsea"] + 1, 32) and c["wn"].shape == c["cg"].shape
    assert [f.shape for f in c["fields"][40:]] == [(30, nsealm), (8, nsealm), (30, nsealm),
                                                   (19, nsealm), (25, nsealm), (10, nsealm)]
    assert np.all(c["dsii"] > 0) and np.all(np.diff(c["sig"]) > 0)
    p = synth.outg_part_case(seed=9)
    nicp = int(p["ipar"][6])
    n1, n2 = p["icprt"][:nicp], p["icprt"][nicp:]
    assert np.all(n2 >= 1) and np.all(n2 + np.maximum(n1, 1) - 1 <= p["ipar"][7])


@needs_ref
@pytest.mark.gpu
def test_outg_device_equals_host_entry(pkg, synth):
    """ww_outg_device on device arrays (torch's stream) gives the fields ww_outg_va gives."""
    import torch

    L = _gpu_lib(pkg)
    L.ww_outg_device.argtypes = [P, I, P, I, P, P, P, I, I] + [P] * 14 + [P, I, P]
    L.ww_outg_device.restype = I
    c = synth.outg_case(seed=11, ste=(1000.0, 1000.0, 3600.0))
    want = _wanted(c)
    f_host = _copy_fields(c["fields"])
    va = np.array(c["va"], copy=True)
    assert call_outg(L, 830, c, f_host, va) == OK
    dev = torch.device("cuda", 0)

    def d(x):
        return torch.from_numpy(np.ascontiguousarray(x)).to(dev)

    arrs = {k: d(c[k]) for k in ("cg", "wn", "dw", "sig", "dden", "dsii", "ecos", "esin", "ec2",
                                 "es2", "esc", "mapsf", "mapsta")}
    d_va = d(c["va"])
    d_f = [d(f) for f in c["fields"]]
    nk, nseal = int(c["ipar"][0]), int(c["ipar"][2])
    ebd = torch.empty(nk * nseal, dtype=torch.float32, device=dev)
    ptrs = (ctypes.c_void_p * 46)(*[t.data_ptr() for t in d_f])
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = L.ww_outg_device(c["ipar"].ctypes.data, 25, c["rpar"].ctypes.data, 10,
                          c["flogrd"].ctypes.data, c["flogr2"].ctypes.data, d_va.data_ptr(),
                          c["va"].shape[1], c["va"].shape[0] - 1,
                          *[arrs[k].data_ptr() for k in ("cg", "wn", "dw", "sig", "dden", "dsii",
                                                          "ecos", "esin", "ec2", "es2", "esc",
                                                          "mapsf", "mapsta")],
                          ebd.data_ptr(), ptrs, 46, stream)
    assert rc == OK
    torch.cuda.synchronize()
    for k in range(46):
        if want[k]:
            assert_bitexact(d_f[k].cpu().numpy(), f_host[k], f"device entry: {NAMES[k]}")
