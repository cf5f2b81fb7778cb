"""The learned DIA surrogate on the GPU: its FP64 judge, its data, its gate, and what training
gains.

- The device FP64 DIA (the judge of every surrogate result) equals the CPU oracle's float64
  restatement of W3SNL1 to 1e-10 of each point's largest term.
- The synthetic sea states equal a float64 numpy restatement of the same draw.
- The gate's fallback is the plain DIA itself: points it rejects carry the plain kernel's bits.
- Training on plain-kernel labels lowers the held-out loss and the error against the FP64 DIA
  many times over the untrained network, and lets the calibrated gate keep points the untrained
  network could not (the gain of the learned part over the method without it: every point on
  the plain DIA).
"""

import numpy as np
import pytest

from conftest import assert_bitexact, cuda_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

IGRID = 41


@pytest.fixture(scope="module")
def sur(pkg):
    import importlib

    pkg.init()
    return importlib.import_module("ww3_gpu_b200.surrogate")


@pytest.fixture(scope="module")
def dia(pkg, synth):
    cfg, sig = synth.dia_config()
    return pkg.Snl1Grid(cfg, sig, igrid=IGRID), cfg, sig


@pytest.fixture(scope="module")
def model(dia, sur):
    return sur.Surrogate(IGRID, nhidden=1024, seed=3)


def _dev(x):
    import torch

    return torch.tensor(np.ascontiguousarray(x), device="cuda")


def _case(synth, n, seed):
    return synth.sea_states(n, seed=seed, depth_range=(5.0, 4000.0), bimodal=0.2)


def test_judge_fp64_matches_cpu_oracle(model, dia, synth, oracle):
    import torch

    _, cfg, sig = dia
    g = _case(synth, 48, seed=21)
    s64 = torch.zeros(48, 1296, dtype=torch.float64, device="cuda")
    d64 = torch.zeros_like(s64)
    stats = torch.zeros(48, 10, dtype=torch.float64, device="cuda")
    model.judge(48, _dev(g["a"]), _dev(g["cg"]), _dev(g["kdmean"]), None, stats, s64, d64)
    torch.cuda.synchronize()
    s_ref, d_ref = oracle.w3snl1_f64(cfg, sig, g["a"], g["cg"], g["kdmean"])
    for got, ref, what in ((s64, s_ref, "S"), (d64, d_ref, "D")):
        got = got.cpu().numpy()
        scale = np.abs(ref).max(axis=1, keepdims=True)
        err = (np.abs(got - ref) / scale).max()
        assert err < 1e-10, f"FP64 {what} differs from the oracle by {err:.2e} of its scale"


def test_judge_of_plain_dia_is_near_zero(model, dia, synth, sur):
    import torch

    grid, _, _ = dia
    g = _case(synth, 256, seed=22)
    s, _ = grid(g["a"], g["cg"], g["kdmean"])
    stats = torch.zeros(256, 10, dtype=torch.float64, device="cuda")
    model.judge(256, _dev(g["a"]), _dev(g["cg"]), _dev(g["kdmean"]), _dev(s), stats)
    e = sur.error_summary(stats.cpu().numpy())
    assert e["hs_tendency_err_max"] < 1e-5
    assert e["s_rel_l2"] < 1e-5
    # Hs as the reference defines it, 4 sqrt(sum A DDEN / CG), against the generator's own Hs.
    hs = stats[:, sur.J_HS].cpu().numpy()
    assert np.allclose(hs, g["hs"], rtol=2e-3)


def _mix64(z):
    z = (z + np.uint64(0x9E3779B97F4A7C15)) & np.uint64(0xFFFFFFFFFFFFFFFF)
    z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & np.uint64(0xFFFFFFFFFFFFFFFF)
    z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & np.uint64(0xFFFFFFFFFFFFFFFF)
    return z ^ (z >> np.uint64(31))


def _uniform(seed, i, j):
    with np.errstate(over="ignore"):
        h = _mix64(_mix64(np.uint64(seed)) ^ ((np.uint64(i) * np.uint64(0x100000001B3) +
                                                np.uint64(j) * np.uint64(0x9E3779B97F4A7C15))
                                               & np.uint64(0xFFFFFFFFFFFFFFFF)))
    return float(h >> np.uint64(11)) * 2.0 ** -53


def test_synthetic_sea_states_match_numpy(model, dia, synth):
    import torch

    _, cfg, sig = dia
    n, seed, p0 = 16, 99, 1000
    a = torch.zeros(n, 1296, device="cuda")
    cg = torch.zeros(n, 36, device="cuda")
    kd = torch.zeros(n, device="cuda")
    model.synth(n, a, cg, kd, seed=seed, bimodal=0.5, dmin=5.0, dmax=4000.0, p0=p0)
    torch.cuda.synchronize()
    s64 = sig.astype(np.float64)
    f = s64 / (2 * np.pi)
    th = np.arange(36) * np.float64(np.float32(cfg["dth"]))
    xfr = np.float64(np.float32(cfg["xfr"]))
    dsii = 0.5 * s64 * (xfr - 1 / xfr)
    for i in range(n):
        u = [_uniform(seed, p0 + i, j) for j in range(10)]
        hs, fp, gam, spr, thm = 0.5 + 7.5 * u[0], 0.06 + 0.14 * u[1], 1 + 4 * u[2], 2 + 18 * u[3], 2 * np.pi * u[4]
        dep = np.exp(np.log(5.0) + (np.log(4000.0) - np.log(5.0)) * u[5])
        swell = u[6] < 0.5
        hs2, fp2, thm2 = 0.5 + 2.5 * u[7], 0.05 + 0.04 * u[8], 2 * np.pi * u[9]

        def jonswap(fpk, gk):
            sg = np.where(f <= fpk, 0.07, 0.09)
            r = np.exp(-(f - fpk) ** 2 / (2 * sg * sg * fpk * fpk))
            return f ** -5 * np.exp(-1.25 * (fpk / f) ** 4) * gk ** r / (2 * np.pi)

        def spread(tm, s):
            return (np.cos(0.5 * (th - tm)) ** 2) ** s

        e1, d1 = jonswap(fp, gam), spread(thm, spr)
        c1 = (hs / 4) ** 2 / (e1 * dsii).sum() / (d1.sum() * th[1])
        e = np.outer(e1, d1) * c1
        if swell:
            e2, d2 = jonswap(fp2, 3.3), spread(thm2, 20.0)
            e = e + np.outer(e2, d2) * (hs2 / 4) ** 2 / (e2 * dsii).sum() / (d2.sum() * th[1])
        k = synth.wavenumber(sig, np.array([dep]))[0]
        kdv = k * dep
        cgv = 0.5 * s64 / k * (1 + 2 * kdv / np.sinh(np.minimum(2 * kdv, 80)))
        aref = e * (cgv / s64)[:, None]
        esum = e.sum(axis=1)
        assert np.allclose(a[i].cpu().numpy().reshape(36, 36), aref, rtol=1e-5, atol=1e-12 * aref.max())
        assert np.allclose(cg[i].cpu().numpy(), cgv, rtol=1e-5)
        assert np.isclose(kd[i].item(), (esum * kdv).sum() / esum.sum(), rtol=1e-5)


def _plain(grid, a, cg, kd, n):
    import torch

    s = torch.zeros(n, 1296, device="cuda")
    d = torch.zeros_like(s)
    grid.run_device(n, a, cg, kd, s, d)
    torch.cuda.synchronize()
    return s.cpu().numpy(), d.cpu().numpy()


def _inputs(model, n, seed):
    import torch

    a = torch.zeros(n, 1296, device="cuda")
    cg = torch.zeros(n, 36, device="cuda")
    kd = torch.zeros(n, device="cuda")
    model.synth(n, a, cg, kd, seed=seed)
    return a, cg, kd


def test_gate_rejecting_everything_is_the_plain_dia(model, dia):
    import torch

    grid, _, _ = dia
    n = 3000
    a, cg, kd = _inputs(model, n, seed=31)
    s = torch.full((n, 1296), float("nan"), device="cuda")
    d = torch.full_like(s, float("nan"))
    acc = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    model.gate(0.0, -1e30)
    model.gated(n, a, cg, kd, s, d, acc)
    assert model.fallback_count() == n
    s_ref, d_ref = _plain(grid, a, cg, kd, n)
    assert_bitexact(s.cpu().numpy(), s_ref, "gated S, all points rejected")
    assert_bitexact(d.cpu().numpy(), d_ref, "gated D, all points rejected")
    assert int(acc.sum()) == 0


def test_gate_accepting_everything_uses_the_network(model, dia):
    import torch

    n = 2000
    a, cg, kd = _inputs(model, n, seed=32)
    s = torch.full((n, 1296), float("nan"), device="cuda")
    d = torch.full_like(s, float("nan"))
    acc = torch.zeros(n, dtype=torch.int32, device="cuda")
    model.gate(1e30, 1e30)
    model.gated(n, a, cg, kd, s, d, acc)
    assert model.fallback_count() == 0
    assert int(acc.sum()) == n
    assert torch.isfinite(s).all()
    assert (d == 0).all()


def test_gate_partial_keeps_plain_bits_on_rejected_points(model, dia):
    import torch

    grid, _, _ = dia
    n = 70000  # two inference chunks
    a, cg, kd = _inputs(model, n, seed=33)
    s = torch.zeros(n, 1296, device="cuda")
    d = torch.zeros_like(s)
    acc = torch.zeros(n, dtype=torch.int32, device="cuda")
    model.gate(0.05, 1e30)
    model.gated(n, a, cg, kd, s, d, acc)
    nrej = model.fallback_count()
    flags = acc.cpu().numpy()
    assert nrej == int((flags == 0).sum())
    s_ref, d_ref = _plain(grid, a, cg, kd, n)
    rej = flags == 0
    if rej.any():
        assert_bitexact(s.cpu().numpy()[rej], s_ref[rej], "rejected points' S")
        assert_bitexact(d.cpu().numpy()[rej], d_ref[rej], "rejected points' D")
    assert (d.cpu().numpy()[~rej] == 0).all()


def _errors(model, sur, n, seed):
    import torch

    a, cg, kd = _inputs(model, n, seed=seed)
    s = torch.zeros(n, 1296, device="cuda")
    d = torch.zeros_like(s)
    model.gate(1e30, 1e30)
    model.gated(n, a, cg, kd, s, d)
    stats = torch.zeros(n, 10, dtype=torch.float64, device="cuda")
    model.judge(n, a, cg, kd, s, stats)
    torch.cuda.synchronize()
    return sur.error_summary(stats.cpu().numpy())


def test_training_gains_over_the_untrained_network(model, sur):
    n_data, holdout = 262144, 16384
    model.dataset(n_data, holdout, seed=5)
    model.loss_weights(1.0, 0.05)
    before_loss = model.eval(n_data - holdout, holdout)
    before = _errors(model, sur, 4096, seed=41)
    cal0 = model.calibrate(8192, seed=42, target=0.02)
    losses = model.train(1500, batch=4096, lr=1e-3, lr_end=1e-5, seed=6)
    after_loss = model.eval(n_data - holdout, holdout)
    after = _errors(model, sur, 4096, seed=41)
    cal1 = model.calibrate(8192, seed=42, target=0.02)
    print(f"held-out MSE {before_loss[0]:.4g} -> {after_loss[0]:.4g}; "
          f"band Hs-tendency error {before['hs_band_err_mean']:.4g} -> "
          f"{after['hs_band_err_mean']:.4g}; S rel L2 {before['s_rel_l2']:.4g} -> "
          f"{after['s_rel_l2']:.4g}; gate keeps {cal0['accepted']:.3f} -> {cal1['accepted']:.3f}")
    assert np.isfinite(losses).all()
    assert after_loss[0] < 0.2 * before_loss[0]
    assert after["s_rel_l2"] < 0.5 * before["s_rel_l2"]
    assert after["hs_band_err_mean"] < 0.5 * before["hs_band_err_mean"]
    assert cal1["accepted"] > cal0["accepted"]
    assert cal1["mean_err_gated"] <= 0.02 + 1e-6


def _gated_device(model, n, a, cg, kd):
    import torch

    s = torch.zeros(n, 1296, device="cuda")
    d = torch.zeros_like(s)
    acc = torch.zeros(n, dtype=torch.int32, device="cuda")
    model.gated(n, a, cg, kd, s, d, acc)
    torch.cuda.synchronize()
    return s, d, acc


@pytest.mark.parametrize("gate", ["open", "few", "many"])
def test_gated_host_entry_equals_device_entry(model, dia, gate):
    """ww_snl1_gated_host (host arrays, copies pipelined over three chunk slots, D cleared on
    the host and only the rejected points' rows copied back) gives the device entry's bits, on a
    batch of three chunks: with no point rejected, with a few (the packed rows), and with more
    than a chunk's packed rows hold (the whole D of such chunks)."""
    import torch

    n = 150_000
    a, cg, kd = _inputs(model, n, seed=34)
    if gate == "open":
        model.gate(1e30, 1e30)
    elif gate == "many":
        model.gate(0.05, 1e30)
    else:
        # a log-error threshold that rejects a few percent of the points (bisection on the
        # device entry's count)
        lo, hi = -50.0, 50.0
        for _ in range(30):
            mid = 0.5 * (lo + hi)
            model.gate(1e30, mid)
            _, _, acc = _gated_device(model, n, a, cg, kd)
            frac = 1.0 - float(acc.float().mean())
            if frac > 0.06:
                lo = mid
            elif frac < 0.01:
                hi = mid
            else:
                break
    s, d, acc = _gated_device(model, n, a, cg, kd)
    nrej = model.fallback_count()
    if gate == "open":
        assert nrej == 0
    elif gate == "few":
        assert 0 < nrej <= n // 8
    h = [t.cpu().pin_memory() for t in (a, cg, kd)]
    hs = torch.full((n, 1296), float("nan")).pin_memory()
    hd = torch.full((n, 1296), float("nan")).pin_memory()
    model.gated_host(n, *h, hs, hd)
    assert model.fallback_count() == nrej
    assert_bitexact(hs.numpy(), s.cpu().numpy(), "host entry S")
    assert_bitexact(hd.numpy(), d.cpu().numpy(), "host entry D")


def test_tma_output_epilogue_equals_row_epilogue(model, dia, monkeypatch):
    """The output layer's two fused epilogues give the same S: tiles of four frequency rows
    rotated in shared memory and stored by TMA (the default) and 256-column tiles stored row by
    row (WW_B200_SUR_EPILOGUE=6). Two inference chunks, the last M tile partial."""
    import torch

    n = 70000
    a, cg, kd = _inputs(model, n, seed=34)
    model.gate(1e30, 1e30)
    out = {}
    for mode in ("6", None):
        if mode:
            monkeypatch.setenv("WW_B200_SUR_EPILOGUE", mode)
        else:
            monkeypatch.delenv("WW_B200_SUR_EPILOGUE", raising=False)
        s = torch.full((n, 1296), float("nan"), device="cuda")
        d = torch.full_like(s, float("nan"))
        acc = torch.zeros(n, dtype=torch.int32, device="cuda")
        model.gated(n, a, cg, kd, s, d, acc)
        torch.cuda.synchronize()
        out[mode] = (s.cpu().numpy(), d.cpu().numpy(), acc.cpu().numpy())
    s6, d6, acc6 = out["6"]
    s7, d7, acc7 = out[None]
    assert np.isfinite(s7).all()
    assert_bitexact(s7, s6, "S, TMA-store epilogue vs row epilogue")
    assert (d7 == 0).all() and (acc7 == acc6).all()
