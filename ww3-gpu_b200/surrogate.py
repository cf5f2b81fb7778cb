"""The learned DIA surrogate's Python mirror (the ww_mlp_* and ww_sur_* entries of libww_b200.so).

The surrogate is this library's own addition (the reference, ww3-gpu, has no learned part): an
MLP trained on the device by the library's tcgen05 kernels on spectra the plain W3SNL1 kernel
labels, used behind a per-point gate whose rejected points go back to the bit-exact DIA. Arrays
are torch tensors on the CUDA device (the entries take device pointers); the classes only
marshal arguments and raise on a non-zero status.
"""

import ctypes

import numpy as np

from . import OK, WwError, init, lib

EPI_GELU_TRAIN, EPI_GELU_INFER, EPI_F32, EPI_DGELU, EPI_ATOMIC = 1, 2, 3, 4, 5
PAIRED = 16  # with EPI_GELU_INFER or EPI_F32: two CTAs of a cluster per 256-row tile

# Per-point columns of ww_sur_judge's statistics.
J_HS, J_TAU_REF, J_TAU_CAND, J_TAU_GROSS, J_BAND_ERR, J_BAND_REF, J_S_ERR2, J_S_REF2, \
    J_FM_REF, J_FM_CAND = range(10)


def _p(x):
    if x is None:
        return None
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    return x.data_ptr()


def _stream(stream):
    if stream is None:
        return None
    return getattr(stream, "cuda_stream", stream)


def gemm(mode, a, b, *, bias=None, out=None, out_t=None, aux=None, out_f32=None, bn=None,
         splits=1, stream=None):
    """C = A . B^T (A: M x K bf16, B: N x K bf16) with epilogue `mode`, through ww_mlp_gemm."""
    init()
    M, K = a.shape
    N = b.shape[0]
    if bn is None:
        bn = next(w for w in (256, 192, 128, 64) if N % w == 0)
    ldo = (out if out is not None else out_f32).shape[1] if (out is not None or out_f32 is not None) else N
    ldt = out_t.shape[1] if out_t is not None else 0
    rc = lib().ww_mlp_gemm(mode, M, N, K, bn, splits, _p(a), a.stride(0), _p(b), b.stride(0),
                           _p(bias), _p(out), _p(out_t), _p(aux), _p(out_f32), ldo, ldt,
                           _stream(stream))
    if rc != OK:
        raise WwError("ww_mlp_gemm", rc)


class Mlp:
    """ww_mlp_*: din -> dh -> dh -> dh -> dout GELU MLP with BF16 weights, FP32 master copy."""

    def __init__(self, din, dh, dout, nvalid=None, cap=256, seed=1):
        init()
        self.L = lib()
        h = ctypes.c_int(0)
        rc = self.L.ww_mlp_create(din, dh, dout, nvalid or dout, cap, seed, ctypes.byref(h))
        if rc != OK:
            raise WwError("ww_mlp_create", rc)
        self.h = h.value
        self.dims = (din, dh, dh, dh, dout)

    def close(self):
        if self.h:
            self.L.ww_mlp_destroy(self.h)
            self.h = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def nparams(self):
        return int(self.L.ww_mlp_param_count(self.h))

    def shapes(self):
        d = self.dims
        return [(d[i + 1], d[i]) for i in range(4)]

    def _split(self, flat):
        out, o = [], 0
        for n, k in self.shapes():
            w = flat[o:o + n * k].reshape(n, k)
            o += n * k
            b = flat[o:o + n]
            o += n
            out.append((w, b))
        return out

    def get_params(self):
        buf = np.empty(self.nparams(), np.float32)
        rc = self.L.ww_mlp_get_params(self.h, buf.ctypes.data)
        if rc != OK:
            raise WwError("ww_mlp_get_params", rc)
        return self._split(buf)

    def set_params(self, layers):
        flat = np.concatenate([np.concatenate([np.ravel(w), np.ravel(b)]) for w, b in layers])
        flat = np.ascontiguousarray(flat, np.float32)
        rc = self.L.ww_mlp_set_params(self.h, flat.ctypes.data)
        if rc != OK:
            raise WwError("ww_mlp_set_params", rc)

    def get_grads(self):
        buf = np.empty(self.nparams(), np.float32)
        rc = self.L.ww_mlp_get_grads(self.h, buf.ctypes.data)
        if rc != OK:
            raise WwError("ww_mlp_get_grads", rc)
        return self._split(buf)

    def train_step(self, x, t, lr=1e-3, wd=0.0, apply=True):
        loss = np.zeros(3, np.float32)
        rc = self.L.ww_mlp_train_step(self.h, x.shape[0], _p(x), _p(t), t.shape[1], lr, wd,
                                      1 if apply else 0, loss.ctypes.data)
        if rc != OK:
            raise WwError("ww_mlp_train_step", rc)
        return loss

    def forward(self, x, out):
        rc = self.L.ww_mlp_forward(self.h, x.shape[0], _p(x), _p(out))
        if rc != OK:
            raise WwError("ww_mlp_forward", rc)
        return out


class Surrogate:
    """ww_sur_*: the surrogate of one DIA grid (the grid's Snl1Grid must exist)."""

    def __init__(self, igrid, nhidden=1024, seed=1):
        init()
        self.L = lib()
        self.igrid = igrid
        self._ok(self.L.ww_sur_init(igrid, nhidden, seed), "ww_sur_init")

    def _ok(self, rc, what):
        if rc != OK:
            raise WwError(what, rc)

    def synth(self, npts, a, cg, kdmean, seed=1, bimodal=0.2, dmin=5.0, dmax=4000.0, p0=0,
              stream=None):
        self._ok(self.L.ww_sur_synth(self.igrid, npts, seed, bimodal, dmin, dmax, p0, _p(a),
                                     _p(cg), _p(kdmean), _stream(stream)), "ww_sur_synth")

    def dataset(self, npts, holdout, seed=1, bimodal=0.2, dmin=5.0, dmax=4000.0):
        self._ok(self.L.ww_sur_dataset(self.igrid, npts, holdout, seed, bimodal, dmin, dmax),
                 "ww_sur_dataset")

    def loss_weights(self, mu, lam):
        self._ok(self.L.ww_sur_loss_weights(self.igrid, mu, lam), "ww_sur_loss_weights")

    def train(self, steps, batch=8192, lr=1e-3, lr_end=1e-5, wd=0.0, seed=1):
        losses = np.zeros((max(steps, 1), 3), np.float32)
        self._ok(self.L.ww_sur_train(self.igrid, steps, batch, lr, lr_end, wd, seed,
                                     losses.ctypes.data), "ww_sur_train")
        return losses[:steps]

    def eval(self, p0, npts):
        loss = np.zeros(3, np.float32)
        self._ok(self.L.ww_sur_eval(self.igrid, p0, npts, loss.ctypes.data), "ww_sur_eval")
        return loss

    def gate(self, energy, log_err):
        self._ok(self.L.ww_sur_gate(self.igrid, energy, log_err), "ww_sur_gate")

    def calibrate(self, npts, seed=7, bimodal=0.2, dmin=5.0, dmax=4000.0, energy=0.05,
                  target=0.02):
        out = np.zeros(4, np.float32)
        self._ok(self.L.ww_sur_calibrate(self.igrid, npts, seed, bimodal, dmin, dmax, energy,
                                         target, out.ctypes.data), "ww_sur_calibrate")
        return {"log_err": float(out[0]), "accepted": float(out[1]),
                "mean_err_gated": float(out[2]), "mean_err_ungated": float(out[3])}

    def gated(self, npts, a, cg, kdmean, s, d, accepted=None, stream=None):
        self.L.ww_snl1_gated(self.igrid, npts, _p(a), _p(cg), _p(kdmean), _p(s), _p(d),
                             _p(accepted), _stream(stream))
        self._ok(self.L.ww_sur_last_error(), "ww_snl1_gated")

    def gated_host(self, npts, a, cg, kdmean, s, d):
        """ww_snl1_gated_host on host arrays (numpy or page-locked torch tensors)."""
        self.L.ww_snl1_gated_host(self.igrid, npts, _p(a), _p(cg), _p(kdmean), _p(s), _p(d))
        self._ok(self.L.ww_sur_last_error(), "ww_snl1_gated_host")

    def forward(self, rows, x, out, stream=None):
        """The network alone on normalised inputs (the four GEMMs of one inference)."""
        self._ok(self.L.ww_sur_forward(self.igrid, rows, _p(x), _p(out), _stream(stream)),
                 "ww_sur_forward")

    def fallback_count(self, stream=None):
        n = self.L.ww_sur_fallback_count(self.igrid, _stream(stream))
        if n < 0:
            raise WwError("ww_sur_fallback_count", self.L.ww_sur_last_error())
        return n

    def judge(self, npts, a, cg, kdmean, s_cand, stats, s64=None, d64=None, stream=None):
        self._ok(self.L.ww_sur_judge(self.igrid, npts, _p(a), _p(cg), _p(kdmean), _p(s_cand),
                                     _p(stats), _p(s64), _p(d64), _stream(stream)),
                 "ww_sur_judge")

    def get_params(self):
        buf = np.empty(int(self.L.ww_sur_param_count(self.igrid)), np.float32)
        self._ok(self.L.ww_sur_get_params(self.igrid, buf.ctypes.data), "ww_sur_get_params")
        return buf

    def set_params(self, flat):
        flat = np.ascontiguousarray(flat, np.float32)
        self._ok(self.L.ww_sur_set_params(self.igrid, flat.ctypes.data), "ww_sur_set_params")


def error_summary(stats):
    """Aggregate ww_sur_judge statistics (npts x 10, numpy float64) into the reported errors of a
    candidate S against the FP64 DIA, per point then averaged:

    - hs_band_err: the band-resolved Hs-tendency error, sum over frequency bands k of
      |tau_k(S) - tau_k(S64)| over sum of |tau_k(S64)|, tau_k = 8/Hs sum_th S DDEN/CG the band's
      share of dHs/dt (Hs = 4 sqrt(sum A DDEN/CG), the reference's W3SRCE definition). The
      gate's error budget. A zero S scores 1.
    - hs_tendency_err: |dHs/dt(S) - dHs/dt(S64)| over the gross tendency 8/Hs sum |S64| DDEN/CG.
      The DIA nearly conserves energy (its net tendency is a few 1e-3 of the gross), so this is
      small even for a poor S; reported, not used to judge.
    - net_hs_tendency_relerr_median: the same difference over |dHs/dt(S64)| itself (median).
    - tm_tendency_relerr_median: relative error of the mean-frequency tendency (median).
    - s_rel_l2: relative L2 error of S over all points and bins."""
    st = np.asarray(stats, np.float64)
    gross = np.where(st[:, J_TAU_GROSS] > 0, st[:, J_TAU_GROSS], np.inf)
    e_hs = np.abs(st[:, J_TAU_CAND] - st[:, J_TAU_REF]) / gross
    band = st[:, J_BAND_ERR] / np.where(st[:, J_BAND_REF] > 0, st[:, J_BAND_REF], np.inf)
    s_l2 = np.sqrt(st[:, J_S_ERR2].sum() / max(st[:, J_S_REF2].sum(), 1e-300))
    net = np.abs(st[:, J_TAU_CAND] - st[:, J_TAU_REF]) / np.maximum(np.abs(st[:, J_TAU_REF]), 1e-300)
    fm = np.abs(st[:, J_FM_CAND] - st[:, J_FM_REF]) / np.maximum(np.abs(st[:, J_FM_REF]), 1e-300)
    return {"hs_band_err_mean": float(band.mean()), "hs_band_err_p90": float(np.quantile(band, 0.9)),
            "hs_band_err_max": float(band.max()),
            "hs_tendency_err_mean": float(e_hs.mean()), "hs_tendency_err_max": float(e_hs.max()),
            "s_rel_l2": float(s_l2),
            "net_hs_tendency_relerr_median": float(np.median(net)),
            "tm_tendency_relerr_median": float(np.median(fm))}
