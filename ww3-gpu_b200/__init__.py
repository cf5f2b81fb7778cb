"""ww3-gpu_b200: the W3SNL1 (DIA) hot path of WAVEWATCH III on B200 behind the reference's C ABI.

The product is ``libww_b200.so`` (ww3-gpu_b200/csrc, CUDA for sm_100a), whose ``extern "C"``
entry points are those the WW3 fork's run-time switch binds in the reference
(ww3-gpu kokkos/src/fortran_iface/ww_kokkos_c.hpp:73-133; declared here in include/ww_b200.h).
This module is the Python mirror of that interface: the same entry names, argument meaning and
status codes, through ctypes, so a test reads like a call from the Fortran side.

There is no CPU fallback: every compute call goes to the CUDA library, and loading fails
loudly when the library is missing or no CUDA device is present.
"""

import ctypes
import os
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "libww_b200.so"
CSRC = HERE / "csrc"

# WwKokkosStatus (ww_kokkos_c.hpp:42-50)
OK = 0
ERR_NOT_INITIALISED = 1
ERR_BAD_SHAPE = 2
ERR_KERNEL = 3
ERR_RUNTIME = 4
ERR_UNSUPPORTED = 5
ERR_TABLE = 6

# ww_snl1_select_kernel choices
KERNEL_AUTO, KERNEL_GATHER, KERNEL_ROWSHIFT, KERNEL_BAND, KERNEL_TILE, KERNEL_PAIR = 0, 1, 2, 3, 4, 5
KERNEL_PAIR_GENERAL = 6

# Every symbol include/ww_b200.h declares.
EXPORTS = (
    "ww_kokkos_init", "ww_kokkos_finalize", "ww_snl1_init", "ww_snl1_init_tables", "ww_snl1",
    "ww_snl1_device", "ww_snl1_enabled", "ww_snl1_last_error", "ww_snl1_select_kernel",
    "ww_kokkos_flag", "ww_kokkos_preset_status", "ww_kokkos_strict", "ww_kokkos_fallback_slot",
    "ww_kokkos_fallback_add", "ww_va_host_read", "ww_va_host_write", "ww_va_host_read_cols",
    "ww_va_host_wrote_cols", "ww_va_host_update", "ww_va_device_zero_cols", "ww_va_device",
    "ww_va_report", "ww_va_device_ptr", "ww_va_state", "ww_steps_fuse", "ww_snl1_autotune",
    "ww_srce_autotune", "ww_autotune_report", "ww_snl1_test_stall", "ww_ktp3_batch", "ww_ktp3_batch_va",
    "ww_prop3_last_error", "ww_xyp3_batch", "ww_xyp3_batch_va", "ww_snl1_noalloc",
    "ww_st4_init", "ww_st4_set_real", "ww_st4_set_int", "ww_st4_commit", "ww_st4_tables", "ww_sds4", "ww_sin4",
    "ww_spr4", "ww_st4_enabled", "ww_st4_last_error", "ww_srce_init", "ww_srce",
    "ww_srce_batch", "ww_srce_batch_va", "ww_srce_enabled", "ww_srce_last_error",
    "ww_srce_batch_device", "ww_xyp3_batch_mpi", "ww_xyp3_mpi_pack", "ww_xyp3_mpi_unpack",
    "ww_map3", "ww_map3_device", "ww_mapt", "ww_utrn", "ww_step_begin", "ww_step_end",
    "ww_step_run", "ww_step_free", "ww_step_ops", "ww_step_nodes", "ww_steps_run", "ww_outg_va", "ww_outg_part",
    "ww_outg_last_error", "ww_outg_device", "ww_wave_gath", "ww_wave_scat", "ww_wave_uwnd",
    "ww_wave_utrn", "ww_wave_dzxy", "ww_wave_map3", "ww_wave_mapt", "ww_wave_distab",
    "ww_wave_cflxy", "ww_snl1_gqm_couple", "ww_snl1_gqm_gauleg", "ww_snl1_gqm_f1f1f1",
    "ww_snl1_gqm_last_error",
    "ww_mlp_create", "ww_mlp_destroy", "ww_mlp_param_count", "ww_mlp_set_params",
    "ww_mlp_get_params", "ww_mlp_get_grads", "ww_mlp_train_step", "ww_mlp_forward",
    "ww_mlp_gemm", "ww_mlp_last_error", "ww_sur_init", "ww_sur_synth", "ww_sur_dataset",
    "ww_sur_loss_weights", "ww_sur_train", "ww_sur_eval", "ww_sur_gate", "ww_sur_calibrate",
    "ww_snl1_gated", "ww_snl1_gated_host", "ww_sur_forward", "ww_sur_fallback_count", "ww_sur_judge", "ww_sur_param_count",
    "ww_sur_get_params", "ww_sur_set_params", "ww_sur_last_error",
)

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_F = ctypes.c_float
_I = ctypes.c_int
_P = ctypes.c_void_p


def build(force=False):
    """Compile libww_b200.so in-tree (nvcc, sm_100a)."""
    if force or not LIB_PATH.exists():
        subprocess.run(["make", "-s", "-C", str(CSRC)], check=True)
    return LIB_PATH


_lib = None


def lib():
    """The loaded C ABI with argument types declared (loads, does not initialise CUDA)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with make -C {CSRC}")
        L = ctypes.CDLL(str(LIB_PATH), mode=ctypes.RTLD_LOCAL)
        L.ww_kokkos_init.argtypes = [_I]
        L.ww_kokkos_init.restype = _I
        L.ww_kokkos_finalize.argtypes = []
        L.ww_kokkos_finalize.restype = None
        L.ww_snl1_init.argtypes = [_I, _I, _I] + [_F] * 10 + [_f32p]
        L.ww_snl1_init.restype = _I
        L.ww_snl1_init_tables.argtypes = [_I, _I, _I] + [_F] * 10 + [_f32p, _i32p, _f32p, _i32p,
                                                                      _i32p, _f32p]
        L.ww_snl1_init_tables.restype = _I
        L.ww_snl1.argtypes = [_I, _I, _P, _P, _P, _P, _P]
        L.ww_snl1.restype = None
        L.ww_snl1_device.argtypes = [_I, _I, _P, _P, _P, _P, _P, _P]
        L.ww_snl1_device.restype = None
        L.ww_snl1_noalloc.argtypes = [_I, _I, _P, _P, _P, _P, _P]
        L.ww_snl1_noalloc.restype = None
        L.ww_st4_init.argtypes = [_I, _P, _I, _P, _I]
        L.ww_st4_init.restype = _I
        L.ww_st4_set_real.argtypes = [_I, _I, _P, _I, _P, _P]
        L.ww_st4_set_real.restype = _I
        L.ww_st4_set_int.argtypes = [_I, _I, _P, _I, _P, _P]
        L.ww_st4_set_int.restype = _I
        L.ww_st4_commit.argtypes = [_I]
        L.ww_st4_commit.restype = _I
        L.ww_sds4.argtypes = [_I, _I] + [_P] * 8 + [_I, _I] + [_P] * 4
        L.ww_sds4.restype = None
        L.ww_sin4.argtypes = [_I, _I] + [_P] * 17
        L.ww_sin4.restype = None
        L.ww_spr4.argtypes = [_I, _I] + [_P] * 20
        L.ww_spr4.restype = None
        L.ww_st4_enabled.argtypes = [_I]
        L.ww_st4_enabled.restype = _I
        L.ww_st4_last_error.restype = _I
        L.ww_srce_init.argtypes = [_I, _P, _I, _P, _I, _P, _P, _P, _P, _P]
        L.ww_srce_init.restype = _I
        L.ww_srce.argtypes = [_I, _I, _I, _I, _I, _P, _P, _P] + [_F] * 8 + [_P] * 26
        L.ww_srce.restype = None
        L.ww_srce_batch.argtypes = [_I, _I, _I, _I, _I, _F, _I] + [_P] * 9
        L.ww_srce_batch.restype = None
        L.ww_srce_batch_va.argtypes = [_I, _I, _I, _I, _I, _F, _P, _I, _I, _I] + [_P] * 9
        L.ww_srce_batch_va.restype = None
        L.ww_srce_enabled.restype = _I
        L.ww_srce_batch_device.argtypes = [_I, _I, _I, _I, _I, _F, _I] + [_P] * 10
        L.ww_srce_batch_device.restype = None
        L.ww_srce_last_error.restype = _I
        L.ww_snl1_enabled.restype = _I
        L.ww_snl1_last_error.restype = _I
        L.ww_snl1_select_kernel.argtypes = [_I, _I]
        L.ww_snl1_select_kernel.restype = _I
        L.ww_kokkos_flag.argtypes = [ctypes.c_char_p]
        L.ww_kokkos_flag.restype = _I
        L.ww_kokkos_preset_status.restype = _I
        L.ww_kokkos_strict.restype = _I
        L.ww_kokkos_fallback_slot.argtypes = [ctypes.c_char_p]
        L.ww_kokkos_fallback_slot.restype = _I
        L.ww_kokkos_fallback_add.argtypes = [_I]
        L.ww_kokkos_fallback_add.restype = None
        for name in ("ww_va_host_read", "ww_va_host_write", "ww_va_host_update"):
            getattr(L, name).argtypes = [_I, _P, _I, _I]
            getattr(L, name).restype = _I
        for name in ("ww_va_host_read_cols", "ww_va_host_wrote_cols", "ww_va_device_zero_cols"):
            getattr(L, name).argtypes = [_I, _P, _I, _I, _I, _P]
            getattr(L, name).restype = _I
        L.ww_va_device.argtypes = [_I, _I]
        L.ww_va_device.restype = _I
        L.ww_va_report.restype = None
        L.ww_va_device_ptr.argtypes = [_I]
        L.ww_va_device_ptr.restype = _P
        L.ww_va_state.argtypes = [_I]
        L.ww_va_state.restype = _I
        L.ww_ktp3_batch.argtypes = [_P, _I, _P, _I] + [_P] * 10 + [_I, _I, _F, _F, _I, _P, _P,
                                                                   _I, _P, _P, _P, _I, _P, _P, _P]
        L.ww_ktp3_batch.restype = _I
        L.ww_ktp3_batch_va.argtypes = [_I, _P, _I, _P, _I] + [_P] * 10 + [
            _I, _I, _F, _F, _I, _P, _P, _I, _P, _P, _P, _P, _I, _I, _P, _P]
        L.ww_ktp3_batch_va.restype = _I
        L.ww_prop3_last_error.restype = _I
        L.ww_xyp3_batch.argtypes = [_P, _I, _P, _I, _P, _I, _P, _I, _F] + [_P] * 21 + [
            _I, _I, _P, _P, _P, _P, _I, _P]
        L.ww_xyp3_batch.restype = _I
        L.ww_xyp3_batch_va.argtypes = [_I, _P, _I, _P, _I, _P, _I, _P, _I, _F] + [_P] * 21 + [
            _I, _I, _P, _P, _P, _P, _P, _I, _I]
        L.ww_xyp3_batch_va.restype = _I
        _LL, _U64 = ctypes.c_longlong, ctypes.c_ulonglong
        L.ww_mlp_create.argtypes = [_I, _I, _I, _I, _I, _U64, ctypes.POINTER(_I)]
        L.ww_mlp_destroy.argtypes = [_I]
        L.ww_mlp_param_count.argtypes = [_I]
        L.ww_mlp_param_count.restype = _LL
        for name in ("ww_mlp_set_params", "ww_mlp_get_params", "ww_mlp_get_grads"):
            getattr(L, name).argtypes = [_I, _P]
        L.ww_mlp_train_step.argtypes = [_I, _I, _P, _P, _I, _F, _F, _I, _P]
        L.ww_mlp_forward.argtypes = [_I, _I, _P, _P]
        L.ww_mlp_gemm.argtypes = [_I, _I, _I, _I, _I, _I, _P, _I, _P, _I] + [_P] * 5 + [_I, _I, _P]
        L.ww_sur_init.argtypes = [_I, _I, _U64]
        L.ww_sur_synth.argtypes = [_I, _I, _U64, _F, _F, _F, _LL, _P, _P, _P, _P]
        L.ww_sur_dataset.argtypes = [_I, _LL, _LL, _U64, _F, _F, _F]
        L.ww_sur_loss_weights.argtypes = [_I, _F, _F]
        L.ww_sur_train.argtypes = [_I, _I, _I, _F, _F, _F, _U64, _P]
        L.ww_sur_eval.argtypes = [_I, _LL, _I, _P]
        L.ww_sur_gate.argtypes = [_I, _F, _F]
        L.ww_sur_calibrate.argtypes = [_I, _I, _U64, _F, _F, _F, _F, _F, _P]
        L.ww_snl1_gated.argtypes = [_I, _I, _P, _P, _P, _P, _P, _P, _P]
        L.ww_snl1_gated.restype = None
        L.ww_snl1_gated_host.argtypes = [_I, _I, _P, _P, _P, _P, _P]
        L.ww_snl1_gated_host.restype = None
        L.ww_sur_fallback_count.argtypes = [_I, _P]
        L.ww_sur_forward.argtypes = [_I, _I, _P, _P, _P]
        L.ww_sur_judge.argtypes = [_I, _I, _P, _P, _P, _P, _P, _P, _P, _P]
        L.ww_sur_param_count.argtypes = [_I]
        L.ww_sur_param_count.restype = _LL
        L.ww_sur_get_params.argtypes = [_I, _P]
        L.ww_sur_set_params.argtypes = [_I, _P]
        for name in ("ww_mlp_create", "ww_mlp_destroy", "ww_mlp_set_params", "ww_mlp_get_params",
                     "ww_mlp_get_grads", "ww_mlp_train_step", "ww_mlp_forward", "ww_mlp_gemm",
                     "ww_mlp_last_error", "ww_sur_init", "ww_sur_synth", "ww_sur_dataset",
                     "ww_sur_loss_weights", "ww_sur_train", "ww_sur_eval", "ww_sur_gate",
                     "ww_sur_calibrate", "ww_sur_fallback_count", "ww_sur_judge",
                     "ww_sur_forward",
                     "ww_sur_get_params", "ww_sur_set_params", "ww_sur_last_error"):
            getattr(L, name).restype = _I
        _lib = L
    return _lib


class WwError(RuntimeError):
    def __init__(self, where, code):
        super().__init__(f"{where} failed with status {code}")
        self.code = code


def init(comm_f=-1):
    """ww_kokkos_init: select the device (WW_KOKKOS_DEVICE_ID) and start the runtime."""
    rc = lib().ww_kokkos_init(comm_f)
    if rc != OK:
        raise WwError("ww_kokkos_init", rc)


def finalize():
    lib().ww_kokkos_finalize()


def last_error():
    return lib().ww_snl1_last_error()


# W3GDATMD's DIA scalars in the order of ww_snl1_init (ww_kokkos_c.hpp:98-100).
SNL1_FIELDS = ("nk", "nth", "xfr", "dth", "lam", "snlc1", "kdcon", "kdmn", "snls1", "snls2",
               "snls3", "fachfe")


def _ptr(x):
    """Data pointer of a C-contiguous numpy array or torch tensor."""
    if isinstance(x, np.ndarray):
        if not x.flags["C_CONTIGUOUS"]:
            raise ValueError("array must be C-contiguous")
        return x.ctypes.data
    if hasattr(x, "data_ptr"):
        if not x.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return x.data_ptr()
    raise TypeError(type(x))


class Snl1Grid:
    """One WW3 grid's W3SNL1 context (the reference's ww_snl1_init / ww_snl1 pair).

    Arrays use the C ABI layout: a (nspec, npts) Fortran array is a C-ordered (npts, nspec)
    array here, (nk, npts) is (npts, nk)."""

    def __init__(self, cfg, sig, igrid=1, tables=None):
        self.L = lib()
        init()
        self.igrid = igrid
        self.cfg = dict(cfg)
        self.nk, self.nth = int(cfg["nk"]), int(cfg["nth"])
        self.nspec = self.nk * self.nth
        args = [cfg[k] for k in SNL1_FIELDS[2:]]
        sig = np.ascontiguousarray(sig, np.float32)
        if tables is None:
            rc = self.L.ww_snl1_init(igrid, self.nk, self.nth, *args, sig)
        else:
            rc = self.L.ww_snl1_init_tables(
                igrid, self.nk, self.nth, *args, sig,
                np.ascontiguousarray(tables["scal"], np.int32),
                np.ascontiguousarray(tables["wts"], np.float32),
                np.ascontiguousarray(tables["ipim"], np.int32),
                np.ascontiguousarray(tables["ic"], np.int32),
                np.ascontiguousarray(tables["af11"], np.float32))
        if rc != OK:
            raise WwError("ww_snl1_init", rc)

    def select_kernel(self, which):
        prev = self.L.ww_snl1_select_kernel(self.igrid, which)
        if prev < 0:
            raise ValueError(f"kernel {which} not available for grid {self.igrid}")
        return prev

    def __call__(self, a, cg, kdmean, s=None, d=None):
        """ww_snl1 on host arrays: copy in, kernel, copy out. Returns (s, d)."""
        a = np.ascontiguousarray(a, np.float32)
        cg = np.ascontiguousarray(cg, np.float32)
        kd = np.ascontiguousarray(kdmean, np.float32)
        npts = a.shape[0] if a.ndim == 2 else 0
        self._check(a, cg, kd, npts)
        s = np.empty_like(a) if s is None else s
        d = np.empty_like(a) if d is None else d
        self.L.ww_snl1(self.igrid, npts, _ptr(a), _ptr(cg), _ptr(kd), _ptr(s), _ptr(d))
        rc = last_error()
        if rc != OK:
            raise WwError("ww_snl1", rc)
        return s, d

    def run_host(self, npts, a, cg, kdmean, s, d):
        """ww_snl1 on caller-owned host buffers (numpy arrays or pinned torch tensors)."""
        self.L.ww_snl1(self.igrid, npts, _ptr(a), _ptr(cg), _ptr(kdmean), _ptr(s), _ptr(d))
        rc = last_error()
        if rc != OK:
            raise WwError("ww_snl1", rc)

    def run_device(self, npts, a, cg, kdmean, s, d, stream=0):
        """ww_snl1_device on device tensors, launched on CUDA stream handle ``stream``."""
        self.L.ww_snl1_device(self.igrid, npts, _ptr(a), _ptr(cg), _ptr(kdmean), _ptr(s),
                              _ptr(d), ctypes.c_void_p(stream))
        rc = last_error()
        if rc != OK:
            raise WwError("ww_snl1_device", rc)

    def _check(self, a, cg, kd, npts):
        if a.ndim != 2 or a.shape[1] != self.nspec:
            raise ValueError(f"a must be (npts, {self.nspec})")
        if cg.shape != (npts, self.nk) or kd.shape != (npts,):
            raise ValueError("cg must be (npts, nk) and kdmean (npts,)")


def flag(name):
    return lib().ww_kokkos_flag(name.encode())


# ---------------------------------------------------------------- ST4 and W3SRCE
def st4_register(igrid, rpar, ipar, regs):
    """ww_st4_init + one ww_st4_set_real/int per (id, array, is_int, lbounds, extents) +
    ww_st4_commit for grid igrid (the sequence W3IOGR / W3KOKKOSMD performs)."""
    L = lib()
    init()
    rpar = np.ascontiguousarray(rpar, np.float32)
    ipar = np.ascontiguousarray(ipar, np.int32)
    rc = L.ww_st4_init(igrid, rpar.ctypes.data, rpar.size, ipar.ctypes.data, ipar.size)
    if rc != OK:
        raise WwError("ww_st4_init", rc)
    for aid, arr, is_int, lb, ext in regs:
        arr = np.ascontiguousarray(arr, np.int32 if is_int else np.float32)
        lb = np.asarray(lb, np.int32)
        ext = np.asarray(ext, np.int32)
        f = L.ww_st4_set_int if is_int else L.ww_st4_set_real
        rc = f(igrid, aid, arr.ctypes.data, len(ext), lb.ctypes.data, ext.ctypes.data)
        if rc != OK:
            raise WwError("ww_st4_set", rc)
    rc = L.ww_st4_commit(igrid)
    if rc != OK:
        raise WwError("ww_st4_commit", rc)


class SrceGrid:
    """One grid's W3SRCE: ST4 registered (st4_register), the DIA (Snl1Grid) and ww_srce_init.
    ``srce`` holds rpar, ipar, sig, dden, ecos, esin, mapwn."""

    def __init__(self, igrid, st4_rpar, st4_ipar, regs, dia_cfg, dia_sig, srce):
        self.L = lib()
        self.igrid = igrid
        st4_register(igrid, st4_rpar, st4_ipar, regs)
        self.dia = Snl1Grid(dia_cfg, dia_sig, igrid=igrid)
        a = {k: np.ascontiguousarray(srce[k]) for k in ("rpar", "ipar", "sig", "dden", "ecos",
                                                          "esin", "mapwn")}
        rc = self.L.ww_srce_init(igrid, a["rpar"].ctypes.data, a["rpar"].size,
                                 a["ipar"].ctypes.data, a["ipar"].size, a["sig"].ctypes.data,
                                 a["dden"].ctypes.data, a["ecos"].ctypes.data,
                                 a["esin"].ctypes.data, a["mapwn"].ctypes.data)
        if rc != OK:
            raise WwError("ww_srce_init", rc)

    def _check(self, who):
        rc = self.L.ww_srce_last_error()
        if rc != OK:
            raise WwError(who, rc)

    def batch(self, npts, spec, wn1, cg1, pin, psc, whitecap, taubbl, tauice, shave, it=1,
              inflags24=0, flogrd57=1, flogrd58=1, dtg=900.0):
        """ww_srce_batch on host buffers (numpy arrays or pinned tensors), updated in place."""
        self.L.ww_srce_batch(self.igrid, it, inflags24, flogrd57, flogrd58, dtg, npts,
                             _ptr(spec), _ptr(wn1), _ptr(cg1), _ptr(pin), _ptr(psc),
                             _ptr(whitecap), _ptr(taubbl), _ptr(tauice), _ptr(shave))
        self._check("ww_srce_batch")

    def batch_va(self, npts, va, jsea, wn1, cg1, pin, psc, whitecap, taubbl, tauice, shave,
                 it=1, inflags24=0, flogrd57=1, flogrd58=1, dtg=900.0):
        """ww_srce_batch_va on the resident VA bound to the host array ``va`` (NSEALM+1 rows of
        NSPEC); jsea (npts, 1-based columns) and the packets are host arrays, updated in place."""
        self.L.ww_srce_batch_va(self.igrid, it, inflags24, flogrd57, flogrd58, dtg, _ptr(va),
                                va.shape[1], va.shape[0] - 1, npts, _ptr(jsea), _ptr(wn1),
                                _ptr(cg1), _ptr(pin), _ptr(psc), _ptr(whitecap), _ptr(taubbl),
                                _ptr(tauice), _ptr(shave))
        self._check("ww_srce_batch_va")

    def batch_device(self, npts, spec, wn1, cg1, pin, psc, whitecap, taubbl, tauice, shave,
                     stream=0, it=1, inflags24=0, flogrd57=1, flogrd58=1, dtg=900.0):
        """ww_srce_batch_device on device tensors, launched on CUDA stream handle ``stream``."""
        self.L.ww_srce_batch_device(self.igrid, it, inflags24, flogrd57, flogrd58, dtg, npts,
                                    _ptr(spec), _ptr(wn1), _ptr(cg1), _ptr(pin), _ptr(psc),
                                    _ptr(whitecap), _ptr(taubbl), _ptr(tauice), _ptr(shave),
                                    ctypes.c_void_p(stream))
        self._check("ww_srce_batch_device")


# ---------------------------------------------------------------- PR3/UQ
KTP3_ARRAYS = ("sig", "dsip", "ecos", "esin", "ec2", "esc", "es2", "mapwn", "mapth2", "mapwn2")


def ktp3_batch(case, itstep=1, ntimes=1, igrid=None, va=None):
    """ww_ktp3_batch (or ww_ktp3_batch_va when ``igrid`` is given, on the resident VA bound to
    the host array ``va``) with the arguments of a dict laid out as the C ABI reads them (see
    synth.ktp3_case). Without ``igrid`` a copy of case["va"] is updated and returned.
    Returns (status, va, cflthmax, cflkmax)."""
    L = lib()
    init()
    rpar = np.ascontiguousarray(case["rpar"], np.float32)
    ipar = np.ascontiguousarray(case["ipar"], np.int32)
    arrs = [np.ascontiguousarray(case[k]) for k in KTP3_ARRAYS]
    cg = np.ascontiguousarray(case["cg"], np.float32)
    wn = np.ascontiguousarray(case["wn"], np.float32)
    js = np.ascontiguousarray(case["jsea"], np.int32)
    isea = np.ascontiguousarray(case["isea"], np.int32)
    ps = np.ascontiguousarray(case["pscal"], np.float32)
    cth = np.array(case["cflthmax"], np.float32, copy=True)
    ck = np.array(case["cflkmax"], np.float32, copy=True)
    head = [rpar.ctypes.data, rpar.size, ipar.ctypes.data, ipar.size] + [a.ctypes.data for a in arrs]
    mid = [itstep, ntimes, case["facth"], case["fack"], case["nsea"], cg.ctypes.data,
           wn.ctypes.data, case["npts"], js.ctypes.data, isea.ctypes.data, ps.ctypes.data]
    if igrid is None:
        v = np.array(case["va"], np.float32, copy=True)
        rc = L.ww_ktp3_batch(*head, *mid, v.shape[0], v.ctypes.data, cth.ctypes.data,
                             ck.ctypes.data)
    else:
        v = va
        rc = L.ww_ktp3_batch_va(igrid, *head, *mid, v.ctypes.data, v.shape[1], v.shape[0] - 1,
                                cth.ctypes.data, ck.ctypes.data)
    return rc, v, cth, ck


def va_host_read(igrid, va):
    """ww_va_host_read on the (NSEALM+1, NSPEC) C-ordered host array bound to grid igrid."""
    return lib().ww_va_host_read(igrid, va.ctypes.data, va.shape[1], va.shape[0] - 1)


def va_host_write(igrid, va):
    return lib().ww_va_host_write(igrid, va.ctypes.data, va.shape[1], va.shape[0] - 1)


XYP3_ARRAYS = ("mapsf", "clats", "sig", "ecos", "esin", "dpdx", "dpdy", "dqdx", "dqdy", "gsqrt",
               "atrnx", "atrny", "mapx2", "mapy2", "mapaxy", "mapcxy", "maptrn", "mapsta", "cg",
               "cx", "cy")


def map3(nx, ny, nsea, nk, nth, mapsta, mapsf, gtype=1, mapth2=None):
    """W3MAP3 through ww_map3: returns (status, dict of mapx2, mapy2, mapaxy, mapcxy, mapth2,
    mapwn2, counts). mapsta is MAPSTA(NY,NX) flattened column-major, mapsf MAPSF(NSEA,3)."""
    L = lib()
    init()
    nxy = nx * ny
    out = {"mapx2": np.zeros(nxy, np.int32), "mapy2": np.zeros(nxy, np.int32),
           "mapaxy": np.zeros(nxy, np.int32), "mapcxy": np.zeros(max(nsea, 1), np.int32),
           "mapth2": (np.zeros((nk + 2) * nth, np.int32) if mapth2 is None
                      else np.array(mapth2, np.int32, copy=True)),
           "mapwn2": np.zeros(nk * nth + nth, np.int32), "counts": np.zeros(8, np.int32)}
    sta = np.ascontiguousarray(mapsta, np.int32)
    sf = np.ascontiguousarray(mapsf, np.int32)
    L.ww_map3.argtypes = [_I] * 6 + [_P] * 9
    L.ww_map3.restype = _I
    rc = L.ww_map3(nx, ny, nsea, nk, nth, gtype, sta.ctypes.data, sf.ctypes.data,
                   *[out[k].ctypes.data for k in ("mapx2", "mapy2", "mapaxy", "mapcxy", "mapth2",
                                                  "mapwn2", "counts")])
    return rc, out


def mapt(nx, ny, nsea, mapsf, atrnx, atrny, maptrn):
    """W3MAPT through ww_mapt; returns (status, maptrn)."""
    L = lib()
    init()
    t = np.array(maptrn, np.int32, copy=True)
    sf = np.ascontiguousarray(mapsf, np.int32)
    ax = np.ascontiguousarray(atrnx, np.float32)
    ay = np.ascontiguousarray(atrny, np.float32)
    L.ww_mapt.argtypes = [_I, _I, _I, _P, _P, _P, _P]
    L.ww_mapt.restype = _I
    rc = L.ww_mapt(nx, ny, nsea, sf.ctypes.data, ax.ctypes.data, ay.ctypes.data, t.ctypes.data)
    return rc, t


def utrn(nx, ny, nsea, trflag, fice0, ficen, ficel, ffacberg, flagll, trny_before, trnx, trny,
         mapsf, mapsta, hpfac, hqfac, ice, berg):
    """W3UTRN through ww_utrn; returns (status, atrnx, atrny), each (3*NX*NY) column-major."""
    L = lib()
    init()
    nxy = nx * ny
    ax = np.zeros(3 * nxy, np.float32)
    ay = np.zeros(3 * nxy, np.float32)
    keep = [np.ascontiguousarray(a, t) for a, t in ((trnx, np.float32), (trny, np.float32),
                                                     (mapsf, np.int32), (mapsta, np.int32),
                                                     (hpfac, np.float32), (hqfac, np.float32),
                                                     (ice, np.float32), (berg, np.float32))]
    L.ww_utrn.argtypes = [_I] * 4 + [_F] * 4 + [_I, _F] + [_P] * 10
    L.ww_utrn.restype = _I
    rc = L.ww_utrn(nx, ny, nsea, trflag, fice0, ficen, ficel, ffacberg, int(flagll),
                   trny_before, *[k.ctypes.data for k in keep], ax.ctypes.data, ay.ctypes.data)
    return rc, ax, ay


class Step:
    """A whole time step of grid ``igrid`` recorded once (ww_step_begin .. ww_step_end) and
    replayed as one CUDA graph (ww_step_run). Use as ``with Step(igrid) as st: <_va calls>``,
    then ``st.run(n)``."""

    def __init__(self, igrid):
        self.L = lib()
        init()
        self.igrid = igrid
        for name in ("ww_step_begin", "ww_step_end", "ww_step_free", "ww_step_ops",
                     "ww_step_nodes"):
            getattr(self.L, name).argtypes = [_I]
            getattr(self.L, name).restype = _I
        self.L.ww_step_run.argtypes = [_I, _I, _P]
        self.L.ww_step_run.restype = _I

    def __enter__(self):
        rc = self.L.ww_step_begin(self.igrid)
        if rc != OK:
            raise WwError("ww_step_begin", rc)
        return self

    def __exit__(self, et, ev, tb):
        rc = self.L.ww_step_end(self.igrid)
        if rc != OK and et is None:
            raise WwError("ww_step_end", rc)
        return False

    def ops(self):
        return self.L.ww_step_ops(self.igrid)

    def nodes(self):
        return self.L.ww_step_nodes(self.igrid)

    def run(self, nrep=1, stream=None):
        rc = self.L.ww_step_run(self.igrid, nrep, stream)
        if rc != OK:
            raise WwError("ww_step_run", rc)

    def free(self):
        self.L.ww_step_free(self.igrid)


def autotune_report():
    """The autotuner's choices so far (ww_autotune_report) as a dict."""
    import json
    L = lib()
    L.ww_autotune_report.argtypes = [ctypes.c_char_p, _I]
    L.ww_autotune_report.restype = _I
    n = L.ww_autotune_report(None, 0)
    if n < 0:
        raise WwError("ww_autotune_report", n)
    buf = ctypes.create_string_buffer(n + 1)
    L.ww_autotune_report(buf, n + 1)
    return json.loads(buf.value.decode())


def snl1_autotune(igrid):
    """ww_snl1_autotune: time the DIA kernels that fit grid igrid, select the fastest."""
    L = lib()
    L.ww_snl1_autotune.argtypes = [_I]
    L.ww_snl1_autotune.restype = _I
    k = L.ww_snl1_autotune(igrid)
    if k < 0:
        raise WwError("ww_snl1_autotune", last_error())
    return k


def srce_autotune(igrid, pts, it=1, dtg=900.0):
    """ww_srce_autotune on the host packets of ``pts`` (as synth.srce_points makes them)."""
    L = lib()
    L.ww_srce_autotune.argtypes = [_I, _I, _I, _I, _I, ctypes.c_float, _I] + [_P] * 8
    L.ww_srce_autotune.restype = _I
    a = {k: np.ascontiguousarray(pts[k], np.float32)
         for k in ("spec", "wn1", "cg1", "pin", "psc", "whitecap", "taubbl", "tauice")}
    n = a["spec"].shape[0]
    c = L.ww_srce_autotune(igrid, it, 0, 1, 1, dtg, n, *[a[k].ctypes.data for k in
                                                          ("spec", "wn1", "cg1", "pin", "psc",
                                                           "whitecap", "taubbl", "tauice")])
    if c < 0:
        raise WwError("ww_srce_autotune", lib().ww_srce_last_error())
    return c


def steps_fuse(igrids):
    """ww_steps_fuse: merge the recorded steps of these grids into one graph with a single W3SRCE
    launch over all their points (an empty list drops it)."""
    L = lib()
    L.ww_steps_fuse.argtypes = [_P, _I]
    L.ww_steps_fuse.restype = _I
    ids = np.ascontiguousarray(igrids, np.int32)
    rc = L.ww_steps_fuse(ids.ctypes.data if ids.size else None, ids.size)
    if rc != OK:
        raise WwError("ww_steps_fuse", rc)


def steps_run(igrids, nrep=1, stream=None):
    """ww_steps_run: the recorded steps of several grids replayed one grid after another (or as
    their fused graph when ww_steps_fuse built one for this list)."""
    L = lib()
    L.ww_steps_run.argtypes = [_P, _I, _I, _P]
    L.ww_steps_run.restype = _I
    ids = np.ascontiguousarray(igrids, np.int32)
    rc = L.ww_steps_run(ids.ctypes.data, ids.size, nrep, stream)
    if rc != OK:
        raise WwError("ww_steps_run", rc)


def xyp3_batch(case, igrid=None, va=None):
    """ww_xyp3_batch (or ww_xyp3_batch_va on the resident VA bound to ``va`` when ``igrid`` is
    given) with a dict of the C ABI's arguments (see synth.xyp3_case). Returns (status, va)."""
    L = lib()
    init()
    keep = {k: np.ascontiguousarray(case[k]) for k in
            ("rpar", "ipar", "imaps", "tscal", "isbpi", "bbpi0", "bbpin", "on") + XYP3_ARRAYS}
    head = [keep["rpar"].ctypes.data, keep["rpar"].size, keep["ipar"].ctypes.data,
            keep["ipar"].size, keep["imaps"].ctypes.data, keep["imaps"].size,
            keep["tscal"].ctypes.data, keep["tscal"].size, case["dtg"]]
    arrs = [keep[k].ctypes.data for k in XYP3_ARRAYS]
    tail = [case["flbpi"], case["nbi"], keep["isbpi"].ctypes.data, keep["bbpi0"].ctypes.data,
            keep["bbpin"].ctypes.data, keep["on"].ctypes.data]
    if igrid is None:
        v = np.array(case["va"], np.float32, copy=True)
        rc = L.ww_xyp3_batch(*head, *arrs, *tail, v.shape[0], v.ctypes.data)
    else:
        v = va
        rc = L.ww_xyp3_batch_va(igrid, *head, *arrs, *tail, v.ctypes.data, v.shape[1],
                                v.shape[0] - 1)
    return rc, v
