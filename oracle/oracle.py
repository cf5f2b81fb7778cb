"""TEST INFRASTRUCTURE ONLY: ctypes access to the CPU oracles of the DIA.

Two checkers, both CPU code, loaded only by tests/, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of bench.py:

* ``liboracle.so`` -- this project's plain-C restatement of INSNL1 and W3SNL1
  (oracle/dia_body.h, following ww3-gpu kokkos/src/ww_kokkos/snl1_tables.cpp:82-329 and
  snl1_team.hpp:351-497), in float32 (bit-exact form) and float64 (the FP64 DIA).
* ``_ref/libref_ww3.so`` -- the reference's own C++ (snl1_tables.cpp, snl1_dia.cpp, the C ABI
  shims snl1_shim.cpp, prop3_shim.cpp and resident_shim.cpp with the headers they include)
  compiled unmodified against oracle/kokkos_compat; present when oracle/Makefile's ``ref``
  target ran where the reference is checked out.

Arrays follow the reference's C ABI: a spectrum batch (nspec, npts) column-major is a numpy
array of shape (npts, nspec) in C order.
"""

import ctypes
import os
import pathlib

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
REF_PATH = HERE / "_ref" / "libref_ww3.so"

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


class Snl1Config(ctypes.Structure):
    """W3GDATMD's DIA scalars in the order of ww::snl1::Config (snl1_config.hpp:54-70)."""

    _fields_ = [("nk", ctypes.c_int), ("nth", ctypes.c_int)] + [
        (n, ctypes.c_float) for n in ("xfr", "dth", "lam", "snlc1", "kdcon", "kdmn", "snls1",
                                      "snls2", "snls3", "fachfe")]

    FIELDS = ("nk", "nth", "xfr", "dth", "lam", "snlc1", "kdcon", "kdmn", "snls1", "snls2",
              "snls3", "fachfe")

    @classmethod
    def from_mapping(cls, m):
        return cls(*[m[k] for k in cls.FIELDS])


def reference_root():
    """Where the reference checkout is: the WW_REFERENCE_ROOT environment variable, else a
    checkout named `reference` beside this repository."""
    env = os.environ.get("WW_REFERENCE_ROOT")
    return pathlib.Path(env) if env else HERE.parent.parent / "reference"


def build():
    """Compile liboracle.so (always) and the reference build (when the reference is present)."""
    import subprocess

    subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True)
    ref = reference_root()
    if (ref / "kokkos/src/ww_kokkos/snl1_team.hpp").exists():
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REF={ref}"], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(LIB_PATH))
        cfgp = ctypes.POINTER(Snl1Config)
        L.oracle_insnl1_f32.argtypes = [cfgp, _f32p, _i32p, _f32p, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        L.oracle_insnl1_f32.restype = ctypes.c_int
        L.oracle_w3snl1_f32.argtypes = [cfgp, _f32p, ctypes.c_int, _f32p, _f32p, _f32p, _f32p,
                                        _f32p, ctypes.c_int, ctypes.c_int]
        L.oracle_w3snl1_f32.restype = ctypes.c_int
        L.oracle_w3snl1_f64.argtypes = [cfgp, _f64p, ctypes.c_int, _f64p, _f64p, _f64p, _f64p,
                                        _f64p, ctypes.c_int]
        L.oracle_w3snl1_f64.restype = ctypes.c_int
        _lib = L
    return _lib


def insnl1(cfg, sig, o0_chain=False):
    """INSNL1 tables: dict(scal, wts, ipim (16, nspecx), ic (16, nspec), af11), 0-based.

    ``o0_chain`` multiplies AF11 = x**11 out as a -O0 gfortran build does (x^3 * x^8), the
    build the reference's golden vector came from; the default is the -O3 power tree."""
    L = lib()
    c = Snl1Config.from_mapping(cfg)
    sig = np.ascontiguousarray(sig, np.float32)
    scal = np.zeros(5, np.int32)
    wts = np.zeros(19, np.float32)
    if L.oracle_insnl1_f32(ctypes.byref(c), sig, scal, wts, None, None, None, int(o0_chain)) != 0:
        raise ValueError("INSNL1 refused the configuration")
    nspecx, nspec = int(scal[3]), cfg["nk"] * cfg["nth"]
    ipim = np.zeros((16, nspecx), np.int32)
    ic = np.zeros((16, nspec), np.int32)
    af11 = np.zeros(nspecx, np.float32)
    L.oracle_insnl1_f32(ctypes.byref(c), sig, scal, wts, ipim.ctypes.data, ic.ctypes.data,
                        af11.ctypes.data, int(o0_chain))
    return {"scal": scal, "wts": wts, "ipim": ipim, "ic": ic, "af11": af11}


def w3snl1(cfg, sig, a, cg, kdmean, nthreads=0, o0_chain=False):
    """W3SNL1 in float32 on (npts, nspec) spectra; returns (s, d)."""
    L = lib()
    c = Snl1Config.from_mapping(cfg)
    a = np.ascontiguousarray(a, np.float32)
    cg = np.ascontiguousarray(cg, np.float32)
    kd = np.ascontiguousarray(kdmean, np.float32)
    s = np.empty_like(a)
    d = np.empty_like(a)
    if L.oracle_w3snl1_f32(ctypes.byref(c), np.ascontiguousarray(sig, np.float32), a.shape[0],
                           a, cg, kd, s, d, nthreads, int(o0_chain)) != 0:
        raise ValueError("W3SNL1 oracle refused the configuration")
    return s, d


def w3snl1_f64(cfg, sig, a, cg, kdmean, nthreads=0):
    """The FP64 DIA: the same algorithm in double precision; returns (s, d) as float64."""
    L = lib()
    c = Snl1Config.from_mapping(cfg)
    a = np.ascontiguousarray(a, np.float64)
    s = np.empty_like(a)
    d = np.empty_like(a)
    if L.oracle_w3snl1_f64(ctypes.byref(c), np.ascontiguousarray(sig, np.float64), a.shape[0],
                           a, np.ascontiguousarray(cg, np.float64),
                           np.ascontiguousarray(kdmean, np.float64), s, d, nthreads) != 0:
        raise ValueError("W3SNL1 oracle refused the configuration")
    return s, d


# ---------------------------------------------------------------- the reference's own build
_ref = None


def ref_available():
    return REF_PATH.exists()


def ref_lib():
    """The reference's C ABI (ww_kokkos_init / ww_snl1_init / ww_snl1) plus ref_snl1_tables."""
    global _ref
    if _ref is None:
        L = ctypes.CDLL(str(REF_PATH), mode=ctypes.RTLD_LOCAL)
        f = ctypes.c_float
        L.ww_kokkos_init.argtypes = [ctypes.c_int]
        L.ww_kokkos_init.restype = ctypes.c_int
        L.ww_snl1_init.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int] + [f] * 10 + [_f32p]
        L.ww_snl1_init.restype = ctypes.c_int
        L.ww_snl1.argtypes = [ctypes.c_int, ctypes.c_int, _f32p, _f32p, _f32p, _f32p, _f32p]
        L.ww_snl1.restype = None
        L.ww_snl1_last_error.restype = ctypes.c_int
        L.ref_snl1_tables.argtypes = [ctypes.c_int, ctypes.c_int] + [f] * 10 + [
            _f32p, _i32p, _f32p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
            ctypes.c_void_p]
        L.ref_snl1_tables.restype = ctypes.c_int
        if L.ww_kokkos_init(-1) != 0:
            raise RuntimeError("reference ww_kokkos_init failed")
        _ref = L
    return _ref


def _cfg_args(cfg):
    return [cfg[k] for k in Snl1Config.FIELDS[2:]]


def ref_tables(cfg, sig):
    L = ref_lib()
    sig = np.ascontiguousarray(sig, np.float32)
    scal = np.zeros(5, np.int32)
    wts = np.zeros(19, np.float32)
    halo = ctypes.c_int(0)
    L.ref_snl1_tables(cfg["nk"], cfg["nth"], *_cfg_args(cfg), sig, scal, wts, None, None, None,
                      ctypes.byref(halo))
    nspecx, nspec = int(scal[3]), cfg["nk"] * cfg["nth"]
    ipim = np.zeros((16, nspecx), np.int32)
    ic = np.zeros((16, nspec), np.int32)
    af11 = np.zeros(nspecx, np.float32)
    L.ref_snl1_tables(cfg["nk"], cfg["nth"], *_cfg_args(cfg), sig, scal, wts, ipim.ctypes.data,
                      ic.ctypes.data, af11.ctypes.data, ctypes.byref(halo))
    return {"scal": scal, "wts": wts, "ipim": ipim, "ic": ic, "af11": af11, "halo": halo.value}


class RefSnl1:
    """The reference's W3SNL1 through its own C ABI (kokkos/src/fortran_iface/ww_kokkos_c.hpp)."""

    def __init__(self, cfg, sig, igrid=1):
        self.L = ref_lib()
        self.igrid = igrid
        self.nspec = cfg["nk"] * cfg["nth"]
        rc = self.L.ww_snl1_init(igrid, cfg["nk"], cfg["nth"], *_cfg_args(cfg),
                                 np.ascontiguousarray(sig, np.float32))
        if rc != 0:
            raise RuntimeError(f"reference ww_snl1_init returned {rc}")

    def __call__(self, a, cg, kdmean, s=None, d=None):
        a = np.ascontiguousarray(a, np.float32)
        s = np.empty_like(a) if s is None else s
        d = np.empty_like(a) if d is None else d
        self.L.ww_snl1(self.igrid, a.shape[0], a, np.ascontiguousarray(cg, np.float32),
                       np.ascontiguousarray(kdmean, np.float32), s, d)
        rc = self.L.ww_snl1_last_error()
        if rc != 0:
            raise RuntimeError(f"reference ww_snl1 failed with status {rc}")
        return s, d


# ---------------------------------------------------------------- W3KTP3 through the reference
KTP3_ARGS = ("rpar", "ipar", "sig", "dsip", "ecos", "esin", "ec2", "esc", "es2", "mapwn",
             "mapth2", "mapwn2")


def _ktp3_setup(L):
    if getattr(L, "_ktp3_ready", False):
        return
    P, I, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
    L.ww_ktp3_batch.argtypes = [P, I, P, I] + [P] * 10 + [I, I, F, F, I, P, P, I, P, P, P, I, P,
                                                          P, P]
    L.ww_ktp3_batch.restype = I
    L._ktp3_ready = True


def ktp3_call(L, case, itstep=1, ntimes=1):
    """ww_ktp3_batch of library L (the reference build or libww_b200) on a synth.ktp3_case
    dict; returns (status, va, cflthmax, cflkmax) as new arrays."""
    _ktp3_setup(L)
    va = np.array(case["va"], np.float32, copy=True)
    cth = np.array(case["cflthmax"], np.float32, copy=True)
    ck = np.array(case["cflkmax"], np.float32, copy=True)
    arrs = [np.ascontiguousarray(case[k]) for k in KTP3_ARGS]
    keep = [np.ascontiguousarray(case[k]) for k in ("cg", "wn", "jsea", "isea", "pscal")]
    rc = L.ww_ktp3_batch(arrs[0].ctypes.data, arrs[0].size, arrs[1].ctypes.data, arrs[1].size,
                         *[a.ctypes.data for a in arrs[2:]], itstep, ntimes, case["facth"],
                         case["fack"], case["nsea"], keep[0].ctypes.data, keep[1].ctypes.data,
                         case["npts"], keep[2].ctypes.data, keep[3].ctypes.data,
                         keep[4].ctypes.data, va.shape[0], va.ctypes.data, cth.ctypes.data,
                         ck.ctypes.data)
    return rc, va, cth, ck


# ---------------------------------------------------------------- W3MAP3 and W3XYP3
def ref_w3map3(nx, ny, nsea, nk, nth, mapsta, mapsf):
    """The reference's W3MAP3 (prop_map3.hpp) on a grid: (mapx2, mapy2, mapaxy, mapcxy, counts)."""
    L = ref_lib()
    P, I = ctypes.c_void_p, ctypes.c_int
    L.ref_w3map3.argtypes = [I, I, I, I, I] + [P] * 9
    L.ref_w3map3.restype = I
    nxy = nx * ny
    out = [np.zeros(nxy, np.int32) for _ in range(3)] + [np.zeros(nsea, np.int32),
                                                         np.zeros((nk + 2) * nth, np.int32),
                                                         np.zeros(nk * nth + nth, np.int32),
                                                         np.zeros(8, np.int32)]
    mapsta = np.ascontiguousarray(mapsta, np.int32)
    mapsf = np.ascontiguousarray(mapsf, np.int32)
    L.ref_w3map3(nx, ny, nsea, nk, nth, mapsta.ctypes.data, mapsf.ctypes.data,
                 *[o.ctypes.data for o in out])
    return out[0], out[1], out[2], out[3], out[6]


def ref_w3map3_all(nx, ny, nsea, nk, nth, mapsta, mapsf, mapth2=None):
    """The reference's W3MAP3 with every output: dict of mapx2, mapy2, mapaxy, mapcxy, mapth2,
    mapwn2, counts (the maps zero-initialised, mapth2 as given or zero)."""
    L = ref_lib()
    P, I = ctypes.c_void_p, ctypes.c_int
    L.ref_w3map3.argtypes = [I, I, I, I, I] + [P] * 9
    L.ref_w3map3.restype = I
    nxy = nx * ny
    out = {"mapx2": np.zeros(nxy, np.int32), "mapy2": np.zeros(nxy, np.int32),
           "mapaxy": np.zeros(nxy, np.int32), "mapcxy": np.zeros(max(nsea, 1), np.int32),
           "mapth2": (np.zeros((nk + 2) * nth, np.int32) if mapth2 is None
                      else np.array(mapth2, np.int32, copy=True)),
           "mapwn2": np.zeros(nk * nth + nth, np.int32), "counts": np.zeros(8, np.int32)}
    sta = np.ascontiguousarray(mapsta, np.int32)
    sf = np.ascontiguousarray(mapsf, np.int32)
    L.ref_w3map3(nx, ny, nsea, nk, nth, sta.ctypes.data, sf.ctypes.data,
                 *[out[k].ctypes.data for k in ("mapx2", "mapy2", "mapaxy", "mapcxy", "mapth2",
                                                "mapwn2", "counts")])
    return out


def ref_w3mapt(nx, ny, nsea, mapsf, atrnx, atrny, maptrn):
    """The reference's W3MAPT; returns MAPTRN."""
    L = ref_lib()
    P, I = ctypes.c_void_p, ctypes.c_int
    L.ref_w3mapt.argtypes = [I, I, I, P, P, P, P]
    L.ref_w3mapt.restype = I
    t = np.array(maptrn, np.int32, copy=True)
    sf = np.ascontiguousarray(mapsf, np.int32)
    ax = np.ascontiguousarray(atrnx, np.float32)
    ay = np.ascontiguousarray(atrny, np.float32)
    L.ref_w3mapt(nx, ny, nsea, sf.ctypes.data, ax.ctypes.data, ay.ctypes.data, t.ctypes.data)
    return t


def ref_w3utrn(nx, ny, nsea, trflag, fice0, ficen, ficel, ffacberg, flagll, trny_before,
               trnx, trny, mapsf, mapsta, hpfac, hqfac, ice, berg):
    """The reference's W3UTRN; returns (atrnx, atrny), each 3*NX*NY column-major."""
    L = ref_lib()
    P, I, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
    L.ref_w3utrn.argtypes = [I] * 4 + [F] * 4 + [I, F] + [P] * 10
    L.ref_w3utrn.restype = I
    nxy = nx * ny
    ax = np.zeros(3 * nxy, np.float32)
    ay = np.zeros(3 * nxy, np.float32)
    keep = [np.ascontiguousarray(a, t) for a, t in ((trnx, np.float32), (trny, np.float32),
                                                     (mapsf, np.int32), (mapsta, np.int32),
                                                     (hpfac, np.float32), (hqfac, np.float32),
                                                     (ice, np.float32), (berg, np.float32))]
    L.ref_w3utrn(nx, ny, nsea, trflag, fice0, ficen, ficel, ffacberg, int(flagll), trny_before,
                 *[k.ctypes.data for k in keep], ax.ctypes.data, ay.ctypes.data)
    return ax, ay


XYP3_ARGS = ("mapsf", "clats", "sig", "ecos", "esin", "dpdx", "dpdy", "dqdx", "dqdy", "gsqrt",
             "atrnx", "atrny", "mapx2", "mapy2", "mapaxy", "mapcxy", "maptrn", "mapsta", "cg",
             "cx", "cy")


def xyp3_call(L, case):
    """ww_xyp3_batch of library L on a synth.xyp3_case dict; returns (status, va)."""
    P, I, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
    L.ww_xyp3_batch.argtypes = [P, I, P, I, P, I, P, I, F] + [P] * 21 + [I, I, P, P, P, P, I, P]
    L.ww_xyp3_batch.restype = I
    va = np.array(case["va"], np.float32, copy=True)
    keep = {k: np.ascontiguousarray(case[k]) for k in
            ("rpar", "ipar", "imaps", "tscal", "isbpi", "bbpi0", "bbpin", "on") + XYP3_ARGS}
    rc = L.ww_xyp3_batch(keep["rpar"].ctypes.data, keep["rpar"].size, keep["ipar"].ctypes.data,
                         keep["ipar"].size, keep["imaps"].ctypes.data, keep["imaps"].size,
                         keep["tscal"].ctypes.data, keep["tscal"].size, case["dtg"],
                         *[keep[k].ctypes.data for k in XYP3_ARGS], case["flbpi"], case["nbi"],
                         keep["isbpi"].ctypes.data, keep["bbpi0"].ctypes.data,
                         keep["bbpin"].ctypes.data, keep["on"].ctypes.data, va.shape[0],
                         va.ctypes.data)
    return rc, va


# ------------------------------------------------------------------ ST4 and W3SRCE through the reference
# ArrayId of the C ABI (kokkos/src/ww_kokkos/st4_arrays.hpp:41-61).
(A_SIG, A_SIG2, A_DSIP, A_DDEN, A_DDEN2, A_ESIN, A_ECOS, A_TH, A_SATWEIGHTS, A_CUMULW, A_DCKI,
 A_QBI, A_SATINDICES, A_IKTAB, A_TAUT, A_TAUHFT, A_TAUHFT2, A_FWTABLE) = range(18)
NKHS, NKD, NDTAB = 2000, 1300, 2000


def _st4_setup(L):
    if getattr(L, "_st4_ready", False):
        return
    P, I, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
    L.ref_st4_tables.argtypes = [P] * 16
    L.ref_st4_tables.restype = I
    L.ww_st4_init.argtypes = [I, P, I, P, I]
    L.ww_st4_init.restype = I
    L.ww_st4_set_real.argtypes = [I, I, P, I, P, P]
    L.ww_st4_set_real.restype = I
    L.ww_st4_set_int.argtypes = [I, I, P, I, P, P]
    L.ww_st4_set_int.restype = I
    L.ww_st4_commit.argtypes = [I]
    L.ww_st4_commit.restype = I
    L.ww_st4_last_error.restype = I
    L.ww_sds4.argtypes = [I, I] + [P] * 8 + [I, I] + [P] * 4
    L.ww_sds4.restype = None
    L.ww_sin4.argtypes = [I, I] + [P] * 17
    L.ww_sin4.restype = None
    L.ww_spr4.argtypes = [I, I] + [P] * 20
    L.ww_spr4.restype = None
    L.ww_srce_init.argtypes = [I, P, I, P, I, P, P, P, P, P]
    L.ww_srce_init.restype = I
    L.ww_srce_batch.argtypes = [I, I, I, I, I, F, I] + [P] * 9
    L.ww_srce_batch.restype = None
    L.ww_srce_last_error.restype = I
    L._st4_ready = True


def _p(x):
    return None if x is None else x.ctypes.data


def st4_tables(st):
    """The ST4 tables of the synthetic grid ``st`` (ww3_gpu_b200.synth.st4_setup) from the
    reference's own INSIN4 and TABU_* (ref_st4_tables), and the DEL* module scalars; rpar gets
    the DEL* written in."""
    L = ref_lib()
    _st4_setup(L)
    ipar = st["ipar"]
    nk, nth, mk, mth, mspec = (int(ipar[0]), int(ipar[1]), int(ipar[3]), int(ipar[4]),
                               int(ipar[5]))
    nsat = 2 * (mth // 2 - 1) + 1
    R = st["R"]
    tabs = float(st["rpar"][R["SINTAILPAR"]]) > 0.5
    tabs2 = tabs and float(st["rpar"][R["TTAUWSHELTER"]]) > 0
    t = {
        "satweights": np.zeros(nsat * mth, np.float32),
        "satindices": np.zeros(nsat * mth, np.int32),
        "iktab": np.zeros(mk * NDTAB, np.int32),
        "dcki": np.zeros(NKHS * NKD, np.float32),
        "qbi": np.zeros(NKHS * NKD, np.float32),
        "cumulw": np.zeros(mspec * mspec, np.float32),
        "taut": np.zeros(201 * 201, np.float32) if tabs else None,
        "tauhft": np.zeros(101 * 201, np.float32) if tabs else None,
        "tauhft2": np.zeros(101 * 201 * 51, np.float32) if tabs2 else None,
    }
    dl = np.zeros(5, np.float32)
    L.ref_st4_tables(_p(st["rpar"]), _p(ipar), _p(st["sig"]), _p(st["dsip"]), _p(st["th"]),
                     _p(st["ecos"]), _p(t["satweights"]), _p(t["satindices"]), _p(t["iktab"]), _p(t["dcki"]),
                     _p(t["qbi"]), _p(t["cumulw"]), _p(t["taut"]), _p(t["tauhft"]),
                     _p(t["tauhft2"]), _p(dl))
    rpar = st["rpar"].copy()
    for j, name in enumerate(("DELUST", "DELALP", "DELTAUW", "DELU", "DELTAIL")):
        rpar[R[name]] = dl[j]
    t["rpar"] = rpar
    t["nsat"] = nsat
    return t


def st4_registrations(st, t):
    """(id, array, is_int, lbounds, extents) of every ST4 array, as ww_st4_set_real/int takes
    them (st4_arrays.hpp:72-81)."""
    ipar = st["ipar"]
    nk, nth, nspec, mk, mth, mspec = [int(v) for v in ipar[:6]]
    nsat = t["nsat"]
    regs = [
        (A_SIG, st["sig"], False, [0], [nk + 2]),
        (A_SIG2, st["sig2"], False, [1], [nspec]),
        (A_DSIP, st["dsip"], False, [0], [nk + 2]),
        (A_DDEN, st["dden"], False, [1], [nk]),
        (A_DDEN2, st["dden2"], False, [1], [nspec]),
        (A_ESIN, st["esin"], False, [1], [nspec + nth]),
        (A_ECOS, st["ecos"], False, [1], [nspec + nth]),
        (A_TH, st["th"], False, [1], [nth]),
        (A_SATWEIGHTS, t["satweights"], False, [1, 1], [nsat, mth]),
        (A_CUMULW, t["cumulw"], False, [1, 1], [mspec, mspec]),
        (A_DCKI, t["dcki"], False, [1, 1], [NKHS, NKD]),
        (A_QBI, t["qbi"], False, [1, 1], [NKHS, NKD]),
        (A_SATINDICES, t["satindices"], True, [1, 1], [nsat, mth]),
        (A_IKTAB, t["iktab"], True, [1, 1], [mk, NDTAB]),
        (A_FWTABLE, st["fwtable"], False, [0], [301]),
    ]
    if t["taut"] is not None:
        regs.append((A_TAUT, t["taut"], False, [0, 0], [201, 201]))
        regs.append((A_TAUHFT, t["tauhft"], False, [0, 0], [101, 201]))
    if t["tauhft2"] is not None:
        regs.append((A_TAUHFT2, t["tauhft2"], False, [0, 0, 0], [101, 201, 51]))
    return regs


def register_st4(init, set_real, set_int, commit, st, t):
    """Configure one ST4 grid through an init/set_real/set_int/commit quadruple with the
    reference's argument lists; returns commit's status."""
    rc = init(_p(t["rpar"]), len(t["rpar"]), _p(st["ipar"]), len(st["ipar"]))
    if rc != 0:
        return rc
    for aid, arr, is_int, lb, ext in st4_registrations(st, t):
        lb = np.asarray(lb, np.int32)
        ext = np.asarray(ext, np.int32)
        f = set_int if is_int else set_real
        rc = f(aid, _p(np.ascontiguousarray(arr)), len(ext), _p(lb), _p(ext))
        if rc != 0:
            return rc
    return commit()


class RefSt4:
    """The reference's ST4 and W3SRCE through its own C ABI, for grid ``igrid``: ww_st4_*,
    ww_sds4 / ww_sin4 / ww_spr4, ww_snl1_init + ww_srce_init + ww_srce_batch. ``scalar_mvec``
    selects the build whose five libmvec loops run scalar glibc powf/expf per lane."""

    def __init__(self, st, t, igrid=1, srce=None, dia=None, scalar_mvec=False):
        path = REF_PATH.parent / ("libref_ww3_scalar.so" if scalar_mvec else "libref_ww3.so")
        self.L = _ref_variant(path)
        _st4_setup(self.L)
        L, g = self.L, igrid
        self.igrid = g
        self.nk, self.nth = int(st["ipar"][0]), int(st["ipar"][1])
        rc = register_st4(lambda *a: L.ww_st4_init(g, *a), lambda *a: L.ww_st4_set_real(g, *a),
                          lambda *a: L.ww_st4_set_int(g, *a), lambda: L.ww_st4_commit(g), st, t)
        if rc != 0:
            raise RuntimeError(f"reference ST4 registration failed: {rc}")
        if dia is not None:
            cfg, sig = dia
            if L.ww_snl1_init(g, cfg["nk"], cfg["nth"], *_cfg_args(cfg),
                              np.ascontiguousarray(sig, np.float32)) != 0:
                raise RuntimeError("reference ww_snl1_init failed")
        if srce is not None:
            rc = L.ww_srce_init(g, _p(srce["rpar"]), len(srce["rpar"]), _p(srce["ipar"]),
                                len(srce["ipar"]), _p(srce["sig"]), _p(srce["dden"]),
                                _p(srce["ecos"]), _p(srce["esin"]), _p(srce["mapwn"]))
            if rc != 0:
                raise RuntimeError(f"reference ww_srce_init returned {rc}")


_ref_variants = {}


def _ref_variant(path):
    """A reference build by path (each loaded once, RTLD_LOCAL) with ww_kokkos_init done."""
    key = str(path)
    if key == str(REF_PATH):
        return ref_lib()
    if key not in _ref_variants:
        L = ctypes.CDLL(key, mode=ctypes.RTLD_LOCAL)
        L.ww_kokkos_init.argtypes = [ctypes.c_int]
        L.ww_kokkos_init.restype = ctypes.c_int
        f = ctypes.c_float
        L.ww_snl1_init.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int] + [f] * 10 + [_f32p]
        L.ww_snl1_init.restype = ctypes.c_int
        if L.ww_kokkos_init(-1) != 0:
            raise RuntimeError("reference ww_kokkos_init failed")
        _ref_variants[key] = L
    return _ref_variants[key]
