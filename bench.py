"""Benchmark of WAVEWATCH III's per-sea-point hot path on B200: sea-point·steps/s at 36x36 bins.

Five workloads (--workload):

* srce (default) -- the full plain source-term step W3SRCE with ST4 (W3SIN4 + W3SDS4 + W3SPR4),
  the DIA (W3SNL1), W3SBT1 and W3SDB1 on 9520 sea points, 36 x 36 float32, DTG = 900 s with
  dynamic substeps (uneven work per point). Spectra: seeded JONSWAP sea states (frequencies
  geometric from 0.0373 Hz, ratio 1.1; 10-degree directions; Hs ~ U(0.5, 8) m, fp ~ U(0.06, 0.2)
  Hz, gamma ~ U(1, 5), cos^2s spreading s ~ U(2, 20)), depths log-uniform in 10-4000 m,
  U10 ~ U(3, 25) m/s from random directions. One step = one ww_srce_batch call over all points,
  every step restarting from the same inputs.
* dia -- W3SNL1 alone on 262,144 deep-water points per GPU (the DIA of the same spectra).

  value  -- device-resident: inputs in HBM, the device entry (ww_srce_batch_device /
            ww_snl1_device) launched on torch's stream, CUDA events around exactly K steps;
            sea-point·steps/s summed over ranks.
  e2e    -- the public host entry (ww_srce_batch / ww_snl1) on page-locked host buffers:
            host->device copies of the step's inputs and device->host copies of its results
            inside every step.
  roofline -- the kernel's algorithmic HBM bytes per point (W3SRCE: 10,928 B = spectrum in and
            out, WN1/CG1, the PIN/PSC packets, WHITECAP/TAUBBL/TAUICE, SHAVE; DIA: 15,700 B) per
            launch over its CUDA-event duration, against MEASURED_PEAKS.json's HBM copy bandwidth.
  cpu_baseline -- the reference's own C++ (oracle/_ref, compiled from its sources) on this
            host's cores on a bounded sample, rank 0 only.

* step -- the resident whole step (config 2's shape at --nx x --ny, default 360 x 180, about
  45,000 sea points; 1440 x 720 is the survey's size): W3KTP3, W3XYP3, W3KTP3 and W3SRCE on the
  resident VA, recorded once and replayed as one CUDA graph per step (ww_step_run); the grid's
  maps from this project's device W3MAP3. e2e uploads the host VA, runs the step and reads the VA
  back, every step.

* multigrid -- config 4's plain form: 16 regional grids of uneven size (sea points log-uniform
  in 5k-400k times --scale, default 1/16), each with its own winds and depths, every grid's
  whole step recorded once and all grids' graphs replayed one after another per step
  (ww_steps_run); the line also gives the replay by one ww_step_run call per grid
  ("sequential").
* outg -- W3OUTG (ww_outg_device on device arrays; e2e: ww_outg_va with the VA newer on the
  host, the grid arrays copied in and the requested fields copied back) on the resident VA of the
  same --nx x --ny grid, every field the device computes requested, space-time extremes on.

--impl reference runs that CPU reference alone, with the same metric and config (for step, on a
grid a quarter of the size in each direction).
Multi-GPU: both workloads are independent per sea point, so each rank runs its own points (weak
scaling) with no collective on the data path; ranks meet only at the timing barriers.
"""

import argparse
import json
import os
import pathlib
import statistics
import subprocess
import sys
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import __graft_entry__ as entry  # noqa: E402

NPTS_PER_GPU = 262144
NK = NTH = 36
BYTES_PER_POINT = 4 * (NK * NTH + NK + 1 + 2 * NK * NTH)  # 15,700
METRIC = "sea-point·steps/s at 36×36 bins: plain DIA vs gated surrogate, same Hs error"
UNIT = "sea-point*steps/s"
WORKLOAD = ("W3SNL1 DIA 36x36 (config 0 spectra: deep-water JONSWAP, d=4000 m), "
            f"{NPTS_PER_GPU} sea points per GPU")
SRCE_NPTS = 9520
SRCE_BYTES_PER_POINT = 4 * (2 * NK * NTH + 2 * NK + 7 + 2 * 22 + 2 * 8 + 1)  # 10,928
SRCE_WORKLOAD = ("W3SRCE + ST4 (W3SIN4, W3SDS4, W3SPR4) + DIA + W3SBT1 + W3SDB1, 36x36, "
                 f"{SRCE_NPTS} sea points per GPU, DTG 900 s with dynamic substeps")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=None)
    p.add_argument("--warmup", type=int, default=None)
    p.add_argument("--impl", choices=["b200", "reference"], default="b200")
    p.add_argument("--workload", choices=["surrogate", "srce", "dia", "step", "outg",
                                          "multigrid"], default="surrogate")
    p.add_argument("--scale", type=float, default=1.0 / 16.0,
                   help="multigrid workload: factor on the 5k-400k sea points of each grid")
    p.add_argument("--nx", type=int, default=360, help="step/outg workloads: grid longitudes")
    p.add_argument("--ny", type=int, default=180, help="step/outg workloads: grid latitudes")
    p.add_argument("--npts", type=int, default=None)
    p.add_argument("--e2e-steps", type=int, default=None)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-autotune", action="store_true",
                   help="skip the autotuner (DIA kernel, W3SRCE CTAs per SM) before timing")
    p.add_argument("--train-steps", type=int, default=30000,
                   help="surrogate workload: AdamW steps of batch 8192 before the timing")
    p.add_argument("--sur-lr", type=float, default=1e-3)
    p.add_argument("--sur-mu", type=float, default=4.0,
                   help="surrogate loss weight of the squared Hs-tendency error")
    p.add_argument("--sur-lambda", type=float, default=0.05,
                   help="surrogate loss weight of the error head")
    p.add_argument("--sur-energy", type=float, default=0.05,
                   help="gate: largest energy residual of an accepted point")
    p.add_argument("--sur-target", type=float, default=0.02,
                   help="gate calibration: mean Hs-tendency error budget")
    p.add_argument("--gate-open", action="store_true",
                   help="surrogate workload: keep every point on the network (no calibration); "
                        "with --train-steps 0 it times the kernels of the network path alone")
    p.add_argument("--no-srce-line", action="store_true",
                   help="surrogate workload: leave out the W3SRCE line it carries")
    p.add_argument("--kernel", choices=["auto", "gather", "rowshift", "band", "tile", "pair", "pair-general"], default="auto",
                   help="DIA kernel (ww_snl1_select_kernel); auto picks the pair kernel")
    a = p.parse_args()
    srce = a.workload == "srce"
    if a.steps is None:
        a.steps = {"surrogate": 50, "srce": 20, "dia": 200, "step": 10, "outg": 20,
                   "multigrid": 5}[a.workload]
    if a.warmup is None:
        a.warmup = 5 if a.workload in ("dia", "surrogate") else 3
    if a.npts is None:
        a.npts = SRCE_NPTS if srce else NPTS_PER_GPU
    return a


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def config(args, world):
    return {"workload": WORKLOAD, "nk": NK, "nth": NTH, "npts_per_gpu": args.npts,
            "global_points": args.npts * world, "depth_m": 4000.0, "seed": 2024,
            "l2": "inputs+outputs 4.1 GB per pass > 126 MB L2 (no flush needed)",
            "parallelism": f"points sharded over {world} GPU(s), no collective"}


# ---------------------------------------------------------------------------- CPU reference
def cpu_reference_rate(cfg, sig, g, seconds=10.0, max_points=4096):
    """Points/s of the reference's C++ on the host cores (its own C ABI, OpenMP over points),
    on a bounded sample of the workload; falls back to the oracle port when the reference
    build is absent. Returns (rate, kind, cores, sample)."""
    oracle = entry.load_oracle()
    n = min(max_points, g["a"].shape[0])
    a, cg, kd = g["a"][:n], g["cg"][:n], g["kdmean"][:n]
    if oracle.ref_available():
        run = oracle.RefSnl1(cfg, sig, igrid=1)
        kind = "reference"
        call = lambda: run(a, cg, kd)  # noqa: E731
    else:
        kind = "port"
        call = lambda: oracle.w3snl1(cfg, sig, a, cg, kd)  # noqa: E731
    call()  # warm-up
    t0 = time.perf_counter()
    calls = 0
    while True:
        call()
        calls += 1
        el = time.perf_counter() - t0
        if el >= seconds or calls >= 200:
            break
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return n * calls / el, kind, cores, f"{calls} calls x {n} points of the workload"


def run_reference_dia(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    entry.load_package()
    synth = __import__("ww3_gpu_b200.synth", fromlist=["synth"])
    cfg, sig = synth.dia_config(NK, NTH)
    n = 2048
    g = synth.sea_states(n, seed=2024, depth=4000.0)
    oracle = entry.load_oracle()
    if oracle.ref_available():
        run = oracle.RefSnl1(cfg, sig, igrid=1)
        kind = "reference"
        step = lambda: run(g["a"], g["cg"], g["kdmean"])  # noqa: E731
    else:
        kind = "port"
        step = lambda: oracle.w3snl1(cfg, sig, g["a"], g["cg"], g["kdmean"])  # noqa: E731
    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    el = time.perf_counter() - t0
    rate = n * args.steps / el
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    cfgd = config(args, 1)
    cfgd["reference_sample_points_per_step"] = n
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": cfgd,
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": f"{n} points of the workload per step, OpenMP over points"},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]
        return False

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------- B200 arm
def measured_peak_hbm():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def ncu_traffic_per_point(kernel_name):
    """DRAM bytes per sea point of kernel `kernel_name` from the committed ncu capture summary
    (profiles/<kernel_name>_36x36.json, or without the _kernel suffix), or None."""
    p = ROOT / "profiles" / f"{kernel_name}_36x36.json"
    if not p.exists():
        p = ROOT / "profiles" / f"{kernel_name.removesuffix('_kernel')}_36x36.json"
    if not p.exists():
        return None
    try:
        j = json.loads(p.read_text())
        return float(j["dram_bytes"]) / float(j["points"])
    except Exception:
        return None


def run_b200_dia(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    rank, world, local = dist_env()
    if not torch.cuda.is_available():
        raise SystemExit("bench.py: no CUDA device; the B200 arm has no CPU fallback")
    torch.cuda.set_device(local)
    os.environ.setdefault("WW_KOKKOS_DEVICE_ID", str(local))
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))

    pkg = entry.load_package()
    synth = __import__("ww3_gpu_b200.synth", fromlist=["synth"])
    cfg, sig = synth.dia_config(NK, NTH)
    npts = args.npts
    g = synth.sea_states_chunked(npts, seed=2024 + rank, depth=4000.0)
    grid = pkg.Snl1Grid(cfg, sig, igrid=1)
    kernel_ids = {"auto": pkg.KERNEL_AUTO, "gather": pkg.KERNEL_GATHER,
                  "rowshift": pkg.KERNEL_ROWSHIFT, "band": pkg.KERNEL_BAND,
                  "tile": pkg.KERNEL_TILE, "pair": pkg.KERNEL_PAIR,
                  "pair-general": pkg.KERNEL_PAIR_GENERAL}
    grid.select_kernel(kernel_ids[args.kernel])
    cur = grid.select_kernel(kernel_ids[args.kernel])  # the kernel that choice resolves to
    if args.kernel == "auto" and not args.no_autotune:
        cur = pkg.snl1_autotune(1)
    kernel_name = {pkg.KERNEL_GATHER: "snl1_gather_kernel", pkg.KERNEL_ROWSHIFT:
                   "snl1_rowshift_kernel", pkg.KERNEL_BAND: "snl1_band_kernel",
                   pkg.KERNEL_TILE: "snl1_tile_kernel", pkg.KERNEL_PAIR: "snl1_pairtile_kernel",
                   pkg.KERNEL_PAIR_GENERAL: "snl1_pair_kernel"}[cur]
    dev = torch.device("cuda", local)
    a = torch.from_numpy(g["a"]).to(dev)
    cg = torch.from_numpy(g["cg"]).to(dev)
    kd = torch.from_numpy(g["kdmean"]).to(dev)
    s = torch.empty_like(a)
    d = torch.empty_like(a)
    stream = torch.cuda.current_stream(dev)
    handle = stream.cuda_stream

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---- device-resident value
    for _ in range(args.warmup):
        grid.run_device(npts, a, cg, kd, s, d, handle)
    barrier()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    with ClockSampler(local) as clk:
        time.sleep(0.3)  # let the sampler start
        barrier()
        ev[0].record(stream)
        for i in range(args.steps):
            grid.run_device(npts, a, cg, kd, s, d, handle)
            ev[i + 1].record(stream)
        barrier()
    per_launch_ms = [ev[i].elapsed_time(ev[i + 1]) for i in range(args.steps)]
    total_ms = max_over_ranks(ev[0].elapsed_time(ev[-1]))
    value = npts * world * args.steps / (total_ms / 1e3)
    launch_ms = sum(per_launch_ms) / len(per_launch_ms)

    # ---- end to end through the host entry, page-locked host buffers
    e2e_steps = args.e2e_steps or max(3, min(args.steps, 10))
    h_a = torch.from_numpy(g["a"]).pin_memory()
    h_cg = torch.from_numpy(g["cg"]).pin_memory()
    h_kd = torch.from_numpy(g["kdmean"]).pin_memory()
    h_s = torch.empty_like(h_a).pin_memory()
    h_d = torch.empty_like(h_a).pin_memory()
    grid.run_host(npts, h_a, h_cg, h_kd, h_s, h_d)  # warm-up (allocates the pipeline slots)
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        grid.run_host(npts, h_a, h_cg, h_kd, h_s, h_d)
    barrier()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e_value = npts * world * e2e_steps / e2e_s
    same = bool(torch.equal(h_s.view(torch.int32), s.cpu().view(torch.int32)))

    peak, peak_kind = measured_peak_hbm()
    achieved = BYTES_PER_POINT * npts / (launch_ms / 1e3) / 1e9
    tpp = ncu_traffic_per_point(kernel_name)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": config(args, world),
        "e2e": {"value": e2e_value, "unit": UNIT,
                "h2d_bytes_per_step": int((h_a.numel() + h_cg.numel() + h_kd.numel()) * 4),
                "d2h_bytes_per_step": int((h_s.numel() + h_d.numel()) * 4),
                "steps": e2e_steps, "host_entry": "ww_snl1", "matches_device_entry": same},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                     "traffic": (tpp * npts if tpp else None),
                     "kernel": kernel_name, "launch_ms": launch_ms,
                     "algorithmic_bytes_per_point": BYTES_PER_POINT},
        "gpu_launches": args.steps,
        "autotune": pkg.autotune_report(),
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, kind, cores, sample = cpu_reference_rate(cfg, sig, g)
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": cores, "kind": kind,
                                "sample": sample}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------- W3SRCE workload
def srce_inputs(synth, npts, seed):
    """The W3SRCE grid (ST4 analytic-tail configuration with this project's own ST4 tables,
    the DIA constants of the workload) and npts seeded points."""
    st = synth.st4_setup(NK, NTH, variant="analytic")
    t = synth.st4_tables_own(st)
    sr = synth.srce_setup(st)
    cfg, sig = synth.dia_config(NK, NTH)
    pts = synth.srce_points(npts, seed=seed, nk=NK, nth=NTH)
    return st, t, sr, cfg, sig, pts


def srce_config(args, world, npts=None):
    npts = npts or args.npts
    return {"workload": SRCE_WORKLOAD, "nk": NK, "nth": NTH, "npts_per_gpu": npts,
            "global_points": npts * world, "dtg_s": 900.0,
            "depth_m": "log-uniform 10-4000", "u10_ms": "U(3, 25)", "seed": 2026,
            "st4": "saturation breaking with the cumulative term, analytic high-frequency tail",
            "l2": ("every step restores its 55 MB of inputs and writes a 256 MB buffer (L2 flush) "
                   "inside the timed region"),
            "parallelism": f"points sharded over {world} GPU(s), no collective"}


SRCE_ARRAYS = ("spec", "wn1", "cg1", "pin", "psc", "whitecap", "taubbl", "tauice")


def cpu_reference_srce(st, t, sr, cfg, sig, pts, seconds=10.0, max_points=1024):
    """Points/s of the reference's W3SRCE (its own C++ and C ABI, OpenMP over points) on this
    host's cores, on a bounded sample of the workload."""
    oracle = entry.load_oracle()
    if not oracle.ref_available():
        return None
    n = min(max_points, pts["spec"].shape[0])
    ref = oracle.RefSt4(st, t, igrid=7, srce=sr, dia=(cfg, sig))
    L = ref.L

    def call():
        a = {k: pts[k][:n].copy() for k in SRCE_ARRAYS}
        sh = __import__("numpy").zeros(n, "int32")
        L.ww_srce_batch(7, 1, 0, 1, 1, 900.0, n, *[a[k].ctypes.data for k in ("spec", "wn1", "cg1",
                        "pin", "psc", "whitecap", "taubbl", "tauice")], sh.ctypes.data)
        if L.ww_srce_last_error() != 0:
            raise RuntimeError("reference ww_srce_batch failed")

    call()
    t0 = time.perf_counter()
    calls = 0
    while True:
        call()
        calls += 1
        el = time.perf_counter() - t0
        if el >= seconds or calls >= 50:
            break
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return n * calls / el, "reference", cores, f"{calls} ww_srce_batch calls x {n} points"


def run_reference_srce(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    entry.load_package()
    synth = __import__("ww3_gpu_b200.synth", fromlist=["synth"])
    n = min(1024, args.npts)
    st, t, sr, cfg, sig, pts = srce_inputs(synth, n, 2026)
    oracle = entry.load_oracle()
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "the reference build "
                          "(oracle/_ref) is absent"}), flush=True)
        return 0
    import numpy as np
    ref = oracle.RefSt4(st, t, igrid=7, srce=sr, dia=(cfg, sig))
    L = ref.L

    def step():
        a = {k: pts[k].copy() for k in SRCE_ARRAYS}
        sh = np.zeros(n, np.int32)
        L.ww_srce_batch(7, 1, 0, 1, 1, 900.0, n, *[a[k].ctypes.data for k in SRCE_ARRAYS],
                        sh.ctypes.data)

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    el = time.perf_counter() - t0
    rate = n * args.steps / el
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    cfgd = srce_config(args, 1)
    cfgd["reference_sample_points_per_step"] = n
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": cfgd,
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": f"{n} points of the workload per step, OpenMP over points"},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_b200_srce(args, quiet=False, npts=None, steps=None, warmup=None, igrid=1):
    """The W3SRCE line; with quiet=True (called from another workload, one GPU) it is returned
    instead of printed, for npts points over steps timed steps on grid igrid."""
    import numpy as np
    import torch
    import torch.distributed as dist

    rank, world, local = dist_env()
    if not torch.cuda.is_available():
        raise SystemExit("bench.py: no CUDA device; the B200 arm has no CPU fallback")
    torch.cuda.set_device(local)
    os.environ.setdefault("WW_KOKKOS_DEVICE_ID", str(local))
    if world > 1 and not quiet:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    pkg = entry.load_package()
    synth = __import__("ww3_gpu_b200.synth", fromlist=["synth"])
    npts = npts or args.npts
    steps = steps or args.steps
    warmup = warmup or args.warmup
    st, t, sr, cfg, sig, pts = srce_inputs(synth, npts, 2026 + rank)
    grid = pkg.SrceGrid(igrid, t["rpar"], st["ipar"], synth.st4_registrations(st, t), cfg, sig, sr)
    if not args.no_autotune:  # W3SRCE's CTAs per SM, timed on a sample of these points
        pkg.srce_autotune(igrid, pts)
    dev = torch.device("cuda", local)
    d0 = {k: torch.from_numpy(pts[k]).to(dev) for k in SRCE_ARRAYS}
    d = {k: v.clone() for k, v in d0.items()}
    shave = torch.zeros(npts, dtype=torch.int32, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > L2
    stream = torch.cuda.current_stream(dev)
    handle = stream.cuda_stream

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if world == 1:
            return x
        tt = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        return float(tt.item())

    def step(ev=None):
        for k in SRCE_ARRAYS:
            if k not in ("wn1", "cg1", "pin"):
                d[k].copy_(d0[k])
        flush.zero_()
        if ev is not None:
            ev[0].record(stream)
        grid.batch_device(npts, d["spec"], d["wn1"], d["cg1"], d["pin"], d["psc"],
                          d["whitecap"], d["taubbl"], d["tauice"], shave, handle)
        if ev is not None:
            ev[1].record(stream)

    for _ in range(warmup):
        step()
    barrier()
    kev = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(steps)]
    t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        time.sleep(0.3)
        barrier()
        t_start.record(stream)
        for i in range(steps):
            step(kev[i])
        t_end.record(stream)
        barrier()
    total_ms = max_over_ranks(t_start.elapsed_time(t_end))
    launch_ms = sum(e[0].elapsed_time(e[1]) for e in kev) / steps
    value = npts * world * steps / (total_ms / 1e3)
    out_dev = {k: d[k].cpu().numpy() for k in ("spec", "psc")}

    # ---- end to end through the host entry ww_srce_batch, page-locked host buffers
    e2e_steps = args.e2e_steps or max(3, min(steps, 5))
    h = {k: torch.from_numpy(pts[k].copy()).pin_memory() for k in SRCE_ARRAYS}
    h_shave = torch.zeros(npts, dtype=torch.int32).pin_memory()

    def host_step():
        for k in ("spec", "psc", "whitecap", "taubbl", "tauice"):
            h[k].copy_(torch.from_numpy(pts[k]))
        grid.batch(npts, h["spec"], h["wn1"], h["cg1"], h["pin"], h["psc"], h["whitecap"],
                   h["taubbl"], h["tauice"], h_shave)

    host_step()
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        host_step()
    barrier()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e_value = npts * world * e2e_steps / e2e_s
    same = bool(np.array_equal(h["spec"].numpy().view(np.int32), out_dev["spec"].view(np.int32))
                and np.array_equal(h["psc"].numpy().view(np.int32),
                                   out_dev["psc"].view(np.int32)))
    per_pt_in = NK * NTH + 2 * NK + 7 + 22 + 4 + 2 + 2 + 1
    per_pt_out = NK * NTH + 22 + 4 + 2 + 2 + 1

    peak, peak_kind = measured_peak_hbm()
    achieved = SRCE_BYTES_PER_POINT * npts / (launch_ms / 1e3) / 1e9
    tpp = ncu_traffic_per_point("srce_kernel")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": steps,
        "warmup": warmup, "ms_per_step": total_ms / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": srce_config(args, world, npts),
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 4 * per_pt_in * npts,
                "d2h_bytes_per_step": 4 * per_pt_out * npts, "steps": e2e_steps,
                "host_entry": "ww_srce_batch", "matches_device_entry": same},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak,
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                     "traffic": (tpp * npts if tpp else None), "kernel": "srce_kernel",
                     "launch_ms": launch_ms,
                     "algorithmic_bytes_per_point": SRCE_BYTES_PER_POINT,
                     "note": ("W3SRCE is bound by FP32 issue and its serial ordered sums, not by "
                              "HBM; the fraction shows how far from the HBM ceiling it runs")},
        "gpu_launches": steps,
        "autotune": pkg.autotune_report(),
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not quiet:
        r = cpu_reference_srce(st, t, sr, cfg, sig, pts)
        if r is not None:
            rate, kind, cores, sample = r
            line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": cores, "kind": kind,
                                    "sample": sample}
    if quiet:
        return line
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------- the resident whole step
STEP_WORKLOAD = ("resident whole step on a {nx}x{ny} lon/lat grid ({nsea} sea points, seeded "
                 "smooth land mask, ~70% sea, boundary and excluded points): W3KTP3, W3XYP3 "
                 "(PR3/UQ), W3KTP3, W3SRCE + ST4 + DIA, 36x36, one CUDA graph per step")
# VA read and written by each of the four parts: the minimum HBM traffic of an unfused step.
STEP_BYTES_PER_POINT = 4 * 2 * 4 * NK * NTH  # 41,472


def step_inputs(synth, map3, nx, ny, seed):
    """A grid's whole-step inputs: the W3SRCE/ST4/DIA configuration of the srce workload, the
    PR3 grid (maps from ``map3``, a W3MAP3), the W3KTP3 arguments and the points' packets."""
    st = synth.st4_setup(NK, NTH, variant="analytic")
    t = synth.st4_tables_own(st)
    sr = synth.srce_setup(st)
    cfg, sig = synth.dia_config(NK, NTH)
    xc = synth.xyp3_case(nx, ny, seed=seed, nk=NK, nth=NTH, ref=map3)
    nsea = xc["nsea"]
    kc = synth.ktp3_case(nsea, seed=seed + 1, nk=NK, nth=NTH, nsea=nsea)
    pts = synth.srce_points(nsea, seed=seed + 2, nk=NK, nth=NTH)
    return st, t, sr, cfg, sig, xc, kc, pts


STEP_PACKETS = ("wn1", "cg1", "pin", "psc", "whitecap", "taubbl", "tauice")


def step_calls(lib_calls, va, kc, xc, pts, nsea):
    """The four calls of one step through ``lib_calls`` (ktp3, xyp3, srce callables)."""
    import numpy as np
    ktp3, xyp3, srce = lib_calls
    jsea = np.arange(1, nsea + 1, dtype=np.int32)
    packets = {k: np.array(pts[k], copy=True) for k in STEP_PACKETS}
    shave = np.zeros(nsea, np.int32)

    def one():
        ktp3(kc, 1, va)
        xyp3(xc, va)
        ktp3(kc, 2, va)
        srce(va, jsea, packets, shave)
    return one


def step_config(args, world, nsea):
    return {"workload": STEP_WORKLOAD.format(nx=args.nx, ny=args.ny, nsea=nsea), "nk": NK,
            "nth": NTH, "nx": args.nx, "ny": args.ny, "nsea_per_gpu": nsea,
            "global_points": nsea * world, "dtg_s": 900.0, "seed": 2026,
            "st4": "saturation breaking with the cumulative term, analytic high-frequency tail",
            "l2": "the resident VA (NSPEC x NSEA floats) is larger than L2",
            "parallelism": f"one grid per GPU ({world}), no collective"}


def run_b200_step(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    rank, world, local = dist_env()
    if not torch.cuda.is_available():
        raise SystemExit("bench.py: no CUDA device; the B200 arm has no CPU fallback")
    torch.cuda.set_device(local)
    os.environ.setdefault("WW_KOKKOS_DEVICE_ID", str(local))
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    pkg = entry.load_package()
    synth = __import__("ww3_gpu_b200.synth", fromlist=["synth"])
    pkg.init()

    def map3(nx, ny, nsea, nk, nth, mapsta, mapsf):  # this project's device W3MAP3
        rc, m = pkg.map3(nx, ny, nsea, nk, nth, mapsta, mapsf)
        if rc != 0:
            raise SystemExit(f"ww_map3 failed ({rc})")
        return m["mapx2"], m["mapy2"], m["mapaxy"], m["mapcxy"][:nsea], m["counts"]

    st, t, sr, cfg, sig, xc, kc, pts = step_inputs(synth, map3, args.nx, args.ny, 2026 + rank)
    nsea = xc["nsea"]
    ig = 1
    grid = pkg.SrceGrid(ig, t["rpar"], st["ipar"], synth.st4_registrations(st, t), cfg, sig, sr)
    va = np.array(xc["va"], np.float32, copy=True)

    def srce(v, jsea, pk, shave):
        grid.batch_va(nsea, v, jsea, pk["wn1"], pk["cg1"], pk["pin"], pk["psc"], pk["whitecap"],
                      pk["taubbl"], pk["tauice"], shave)

    va0 = np.array(va, copy=True)
    L = pkg.lib()
    calls = (lambda c, it, v: pkg.ktp3_batch(c, it, 1, ig, v),
             lambda c, v: pkg.xyp3_batch(c, ig, v), srce)

    def fresh_step():
        """The step recorded from the initial state: VA and per-point packets as generated, so
        the device-timed run and the end-to-end run time the same steps."""
        if L.ww_va_state(ig) >= 0:  # the host takes the VA back before it writes it
            assert L.ww_va_host_write(ig, va.ctypes.data, va.shape[1], va.shape[0] - 1) == 0
        va[...] = va0
        st_ = pkg.Step(ig)
        with st_:
            step_calls(calls, va, kc, xc, pts, nsea)()
        return st_

    step = fresh_step()
    nodes = step.nodes()
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    handle = stream.cuda_stream

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if world == 1:
            return x
        tt = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        return float(tt.item())

    for _ in range(args.warmup):
        step.run(1, handle)
    barrier()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    with ClockSampler(local) as clk:
        time.sleep(0.3)
        barrier()
        ev[0].record(stream)
        for i in range(args.steps):
            step.run(1, handle)
            ev[i + 1].record(stream)
        barrier()
    total_ms = max_over_ranks(ev[0].elapsed_time(ev[-1]))
    per = [ev[i].elapsed_time(ev[i + 1]) for i in range(args.steps)]
    value = nsea * world * args.steps / (total_ms / 1e3)

    # ---- end to end: the same steps from the same initial state (re-recorded), with the host
    # VA uploaded before and read back after every step
    e2e_steps = args.steps
    step.free()
    step = fresh_step()
    hva = va  # the Fortran array the resident VA mirrors

    def host_step():
        assert L.ww_va_host_write(ig, hva.ctypes.data, hva.shape[1], hva.shape[0] - 1) == 0
        step.run(1, None)
        assert L.ww_va_host_read(ig, hva.ctypes.data, hva.shape[1], hva.shape[0] - 1) == 0

    for _ in range(args.warmup):
        step.run(1, None)
    assert L.ww_va_host_read(ig, hva.ctypes.data, hva.shape[1], hva.shape[0] - 1) == 0
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        host_step()
    barrier()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e_value = nsea * world * e2e_steps / e2e_s
    va_bytes = int(va.nbytes)
    peak, peak_kind = measured_peak_hbm()
    step_ms = statistics.median(per)
    achieved = STEP_BYTES_PER_POINT * nsea / (step_ms / 1e3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": step_config(args, world, nsea),
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": va_bytes,
                "d2h_bytes_per_step": va_bytes, "steps": e2e_steps,
                "host_entry": "ww_va_host_write + ww_step_run + ww_va_host_read"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak,
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                     "traffic": None, "kernel": "the step graph (srce_kernel dominant)",
                     "launch_ms": step_ms, "algorithmic_bytes_per_point": STEP_BYTES_PER_POINT,
                     "note": ("the VA read and written by each of the four parts; W3SRCE, about "
                              "95% of the step, is bound by its serial chains, not by HBM")},
        "gpu_launches": nodes * args.steps,
        "graph_nodes": nodes,
        "per_step_ms": [round(x, 3) for x in per],
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r = cpu_reference_step(synth, max(args.nx // 4, 8), max(args.ny // 4, 8))
        if r is not None:
            rate, kind, cores, sample = r
            line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": cores, "kind": kind,
                                    "sample": sample}
    if rank == 0:
        print(json.dumps(line), flush=True)
    step.free()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def reference_step_calls(oracle, synth, nx, ny, igrid):
    """The reference's four calls of a whole step (its C ABI, resident VA in host memory) on an
    nx x ny grid of the workload; returns (callable one step, nsea)."""
    import numpy as np
    st, t, sr, cfg, sig, xc, kc, pts = step_inputs(synth, oracle.ref_w3map3, nx, ny, 2026)
    nsea = xc["nsea"]
    ref = oracle.RefSt4(st, t, igrid=igrid, srce=sr, dia=(cfg, sig))
    L = ref.L
    va = np.array(xc["va"], np.float32, copy=True)
    K = ("sig", "dsip", "ecos", "esin", "ec2", "esc", "es2", "mapwn", "mapth2", "mapwn2")
    X = ("mapsf", "clats", "sig", "ecos", "esin", "dpdx", "dpdy", "dqdx", "dqdy", "gsqrt",
         "atrnx", "atrny", "mapx2", "mapy2", "mapaxy", "mapcxy", "maptrn", "mapsta", "cg", "cx",
         "cy")
    kk = {k: np.ascontiguousarray(v) for k, v in kc.items() if isinstance(v, np.ndarray)}
    xk = {k: np.ascontiguousarray(v) for k, v in xc.items() if isinstance(v, np.ndarray)}
    cth = np.array(kc["cflthmax"], np.float32, copy=True)
    ck = np.array(kc["cflkmax"], np.float32, copy=True)

    def ktp3(c, it, v):
        L.ww_ktp3_batch_va(igrid, kk["rpar"].ctypes.data, kk["rpar"].size, kk["ipar"].ctypes.data,
                           kk["ipar"].size, *[kk[a].ctypes.data for a in K], it, 1, c["facth"],
                           c["fack"], c["nsea"], kk["cg"].ctypes.data, kk["wn"].ctypes.data,
                           c["npts"], kk["jsea"].ctypes.data, kk["isea"].ctypes.data,
                           kk["pscal"].ctypes.data, v.ctypes.data, v.shape[1], v.shape[0] - 1,
                           cth.ctypes.data, ck.ctypes.data)

    def xyp3(c, v):
        L.ww_xyp3_batch_va(igrid, xk["rpar"].ctypes.data, xk["rpar"].size, xk["ipar"].ctypes.data,
                           xk["ipar"].size, xk["imaps"].ctypes.data, xk["imaps"].size,
                           xk["tscal"].ctypes.data, xk["tscal"].size, c["dtg"],
                           *[xk[a].ctypes.data for a in X], c["flbpi"], c["nbi"],
                           xk["isbpi"].ctypes.data, xk["bbpi0"].ctypes.data,
                           xk["bbpin"].ctypes.data, xk["on"].ctypes.data, v.ctypes.data,
                           v.shape[1], v.shape[0] - 1)

    def srce(v, jsea, pk, shave):
        L.ww_srce_batch_va(igrid, 1, 0, 1, 1, 900.0, v.ctypes.data, v.shape[1], v.shape[0] - 1,
                           nsea, jsea.ctypes.data, *[pk[k].ctypes.data for k in STEP_PACKETS],
                           shave.ctypes.data)

    c_int, c_float, c_void = (__import__("ctypes").c_int, __import__("ctypes").c_float,
                              __import__("ctypes").c_void_p)
    L.ww_ktp3_batch_va.argtypes = [c_int, c_void, c_int, c_void, c_int] + [c_void] * 10 + [
        c_int, c_int, c_float, c_float, c_int, c_void, c_void, c_int, c_void, c_void, c_void,
        c_void, c_int, c_int, c_void, c_void]
    L.ww_xyp3_batch_va.argtypes = [c_int, c_void, c_int, c_void, c_int, c_void, c_int, c_void,
                                   c_int, c_float] + [c_void] * 21 + [
        c_int, c_int, c_void, c_void, c_void, c_void, c_void, c_int, c_int]
    L.ww_srce_batch_va.argtypes = [c_int, c_int, c_int, c_int, c_int, c_float, c_void, c_int,
                                   c_int, c_int] + [c_void] * 9
    return step_calls((ktp3, xyp3, srce), va, kc, xc, pts, nsea), nsea


def cpu_reference_step(synth, nx, ny, seconds=10.0):
    """Sea-point·steps/s of the reference's whole step on this host's cores, on a smaller grid
    of the workload (its own C++, the resident VA in host memory)."""
    oracle = entry.load_oracle()
    if not oracle.ref_available():
        return None
    one, nsea = reference_step_calls(oracle, synth, nx, ny, 8)
    one()
    t0 = time.perf_counter()
    n = 0
    while True:
        one()
        n += 1
        el = time.perf_counter() - t0
        if el >= seconds or n >= 20:
            break
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return (nsea * n / el, "reference", cores,
            f"{n} whole steps of a {nx}x{ny} grid of the workload ({nsea} sea points)")


def run_reference_step(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    entry.load_package()
    synth = __import__("ww3_gpu_b200.synth", fromlist=["synth"])
    oracle = entry.load_oracle()
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "the reference build "
                          "(oracle/_ref) is absent"}), flush=True)
        return 0
    nx, ny = max(args.nx // 4, 8), max(args.ny // 4, 8)
    one, nsea = reference_step_calls(oracle, synth, nx, ny, 9)
    for _ in range(args.warmup):
        one()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        one()
    el = time.perf_counter() - t0
    rate = nsea * args.steps / el
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    cfgd = step_config(args, 1, nsea)
    cfgd["reference_sample_grid"] = f"{nx}x{ny}"
    sample = f"whole steps of a {nx}x{ny} grid of the workload ({nsea} sea points)"
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": cfgd,
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------------ multi-grid workload
MULTI_NGRIDS = 16
MULTI_WORKLOAD = ("{ngrids} regional grids of uneven size (sea points log-uniform in {lo}-{hi}, "
                  "seeded; {total} in all), each with its own wind field and depth, 36x36: every "
                  "grid's resident whole step (W3KTP3, W3XYP3, W3KTP3, W3SRCE + ST4 + DIA) "
                  "recorded once, the grids' steps fused into one CUDA graph with ONE persistent "
                  "W3SRCE launch over all grids' points (ww_steps_fuse, one work queue), replayed "
                  "once per step (ww_steps_run)")


def multi_shapes(scale, seed=2026):
    """(nx, ny) of each grid: sea points log-uniform in [5000, 400000] * scale, on a 2:1 lon/lat
    grid whose smooth land mask leaves about 70 % sea."""
    import numpy as np
    rng = np.random.default_rng(seed)
    target = np.exp(rng.uniform(np.log(5000.0), np.log(400000.0), MULTI_NGRIDS)) * scale
    shapes = []
    for n in target:
        ny = max(8, int(round((n / 0.7 / 2.0) ** 0.5)))
        shapes.append((2 * ny, ny))
    return shapes


def run_b200_multigrid(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    rank, world, local = dist_env()
    if not torch.cuda.is_available():
        raise SystemExit("bench.py: no CUDA device; the B200 arm has no CPU fallback")
    torch.cuda.set_device(local)
    os.environ.setdefault("WW_KOKKOS_DEVICE_ID", str(local))
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    pkg = entry.load_package()
    synth = __import__("ww3_gpu_b200.synth", fromlist=["synth"])
    pkg.init()

    def map3(nx, ny, nsea, nk, nth, mapsta, mapsf):  # this project's device W3MAP3
        rc, m = pkg.map3(nx, ny, nsea, nk, nth, mapsta, mapsf)
        if rc != 0:
            raise SystemExit(f"ww_map3 failed ({rc})")
        return m["mapx2"], m["mapy2"], m["mapaxy"], m["mapcxy"][:nsea], m["counts"]

    shapes = multi_shapes(args.scale, 2026 + rank)
    grids = []
    for k, (nx, ny) in enumerate(shapes):
        ig = 100 + k
        st, t, sr, cfg, sig, xc, kc, pts = step_inputs(synth, map3, nx, ny, 3000 + 17 * k + rank)
        nsea = xc["nsea"]
        grid = pkg.SrceGrid(ig, t["rpar"], st["ipar"], synth.st4_registrations(st, t), cfg, sig,
                            sr)
        va = np.array(xc["va"], np.float32, copy=True)

        def srce(v, jsea, pk, shave, grid=grid, nsea=nsea):
            grid.batch_va(nsea, v, jsea, pk["wn1"], pk["cg1"], pk["pin"], pk["psc"],
                          pk["whitecap"], pk["taubbl"], pk["tauice"], shave)

        calls = (lambda c, it, v, ig=ig: pkg.ktp3_batch(c, it, 1, ig, v),
                 lambda c, v, ig=ig: pkg.xyp3_batch(c, ig, v), srce)
        grids.append({"ig": ig, "nsea": nsea, "va": va, "va0": np.array(va, copy=True),
                      "calls": calls, "inputs": (kc, xc, pts), "step": None, "grid": grid,
                      "nx": nx, "ny": ny})
    igs = [g["ig"] for g in grids]
    L = pkg.lib()

    def record_all():
        """Every grid's step recorded from its initial VA and packets, so each variant times
        the same steps."""
        for g in grids:
            if g["step"] is not None:
                g["step"].free()
            v = g["va"]
            if L.ww_va_state(g["ig"]) >= 0:  # the host takes the VA back before it writes it
                assert L.ww_va_host_write(g["ig"], v.ctypes.data, v.shape[1], v.shape[0] - 1) == 0
            v[...] = g["va0"]
            kc, xc, pts = g["inputs"]
            step = pkg.Step(g["ig"])
            with step:
                step_calls(g["calls"], v, kc, xc, pts, g["nsea"])()
            g["step"] = step
    total = sum(g["nsea"] for g in grids)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    handle = stream.cuda_stream

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if world == 1:
            return x
        tt = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        return float(tt.item())

    def timed(fn, steps):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
        barrier()
        ev[0].record(stream)
        for i in range(steps):
            fn()
            ev[i + 1].record(stream)
        barrier()
        return max_over_ranks(ev[0].elapsed_time(ev[-1])), [
            ev[i].elapsed_time(ev[i + 1]) for i in range(steps)]

    together = lambda: pkg.steps_run(igs, 1, handle)  # noqa: E731

    if not args.no_autotune:  # W3SRCE's CTAs per SM on the first grid's points (one layout)
        pkg.srce_autotune(grids[0]["ig"], grids[0]["inputs"][2])
    # The grids' graphs one after another (the unfused form), from the initial state.
    record_all()
    pkg.steps_fuse([])
    for _ in range(args.warmup):
        together()
    seq_ms, _ = timed(together, args.steps)
    seq_value = total * world * args.steps / (seq_ms / 1e3)
    # The fused graph: one W3SRCE launch over all grids' points, the same steps.
    record_all()
    pkg.steps_fuse(igs)
    for _ in range(args.warmup):
        together()
    barrier()
    with ClockSampler(local) as clk:
        time.sleep(0.3)
        total_ms, per = timed(together, args.steps)
    value = total * world * args.steps / (total_ms / 1e3)

    # ---- end to end: the same steps again from the initial state, every grid's host VA
    # uploaded, the fused step, every VA read back
    record_all()
    pkg.steps_fuse(igs)
    for _ in range(args.warmup):
        together()
    for g in grids:
        v = g["va"]
        assert L.ww_va_host_read(g["ig"], v.ctypes.data, v.shape[1], v.shape[0] - 1) == 0
    e2e_steps = args.steps

    def host_step():
        for g in grids:
            v = g["va"]
            assert L.ww_va_host_write(g["ig"], v.ctypes.data, v.shape[1], v.shape[0] - 1) == 0
        pkg.steps_run(igs, 1, None)
        for g in grids:
            v = g["va"]
            assert L.ww_va_host_read(g["ig"], v.ctypes.data, v.shape[1], v.shape[0] - 1) == 0

    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        host_step()
    barrier()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    va_bytes = int(sum(g["va"].nbytes for g in grids))
    peak, peak_kind = measured_peak_hbm()
    step_ms = statistics.median(per)
    achieved = STEP_BYTES_PER_POINT * total / (step_ms / 1e3) / 1e9
    lo, hi = int(5000 * args.scale), int(400000 * args.scale)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": MULTI_WORKLOAD.format(ngrids=len(grids), lo=lo, hi=hi,
                                                     total=total),
                   "nk": NK, "nth": NTH, "ngrids": len(grids), "scale": args.scale,
                   "grids": [[g["nx"], g["ny"], g["nsea"]] for g in grids],
                   "sea_points_per_gpu": total, "dtg_s": 900.0,
                   "source_terms": "plain DIA (the surrogate is not used inside W3SRCE)",
                   "l2": "the grids' resident VAs together are larger than L2",
                   "parallelism": f"all grids on each GPU ({world}), no collective"},
        "unfused": {"value": seq_value, "unit": UNIT, "steps": args.steps,
                    "ms_per_step": seq_ms / args.steps,
                    "note": ("the same steps from the same initial state, the grids' recorded "
                             "graphs replayed one after another (one W3SRCE launch per grid)")},
        "fused_speedup": seq_ms / total_ms,
        "e2e": {"value": total * world * e2e_steps / e2e_s, "unit": UNIT,
                "h2d_bytes_per_step": va_bytes, "d2h_bytes_per_step": va_bytes,
                "steps": e2e_steps,
                "host_entry": "ww_va_host_write + ww_steps_run + ww_va_host_read"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak,
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                     "traffic": None, "kernel": "the fused step graph (srce_multi_kernel dominant)",
                     "launch_ms": step_ms, "algorithmic_bytes_per_point": STEP_BYTES_PER_POINT},
        "gpu_launches": (sum(g["step"].nodes() for g in grids) - 2 * len(grids) + 2) * args.steps,
        "autotune": pkg.autotune_report(),
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r = cpu_reference_step(synth, 90, 45)
        if r is not None:
            rate, kind, cores, sample = r
            line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": cores, "kind": kind,
                                    "sample": sample + " (per-point cost does not depend on the "
                                    "grid split)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    for g in grids:
        g["step"].free()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_reference_multigrid(args):
    """The reference's own four calls per step on a 90 x 45 grid of the workload (its per-point
    cost does not depend on how the points are split into grids), reported under the
    multi-grid workload's name."""
    rank, _, _ = dist_env()
    if rank != 0:
        return 0
    import contextlib
    import io
    a = argparse.Namespace(**vars(args))
    a.nx, a.ny = 360, 180
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        rc = run_reference_step(a)
    line = json.loads(buf.getvalue().strip().splitlines()[-1])
    if "config" in line:
        line["config"]["workload"] = ("the multi-grid workload's per-point cost: " +
                                      line["config"]["workload"])
        line["config"]["scale"] = args.scale
    print(json.dumps(line), flush=True)
    return rc


# ---------------------------------------------------------------------------- W3OUTG workload
OUTG_WORKLOAD = ("W3OUTG (ww_outg_va: sections 1-4 and the space-time extremes, every field "
                 "the device computes requested) on the resident VA of a {nx}x{ny} grid "
                 "({nsea} sea points), 36x36")
OUTG_STE = (1000.0, 1000.0, 3600.0)


def outg_bytes_per_point(c):
    """The algorithmic HBM bytes of one sea point of W3OUTG: its VA column, CG and WN (NK+2
    each), DW, MAPSF, MAPSTA, and every field it writes (40 + the 2-D fields' columns)."""
    nk, nth = int(c["ipar"][0]), int(c["ipar"][1])
    ncol = sum(f.shape[0] for f in c["fields"][40:])
    return 4 * (nk * nth + 2 * (nk + 2) + 1 + 3 + 1 + 40 + ncol)


def outg_config(args, world, c):
    return {"workload": OUTG_WORKLOAD.format(nx=args.nx, ny=args.ny, nsea=c["nsea"]),
            "nk": NK, "nth": NTH, "nx": args.nx, "ny": args.ny, "nsea_per_gpu": c["nsea"],
            "global_points": c["nsea"] * world, "seed": 2026,
            "space_time_extremes": {"stexu": OUTG_STE[0], "steyu": OUTG_STE[1],
                                    "stedu": OUTG_STE[2]},
            "l2": "the resident VA (NSPEC x NSEA floats) is larger than L2",
            "parallelism": f"one grid per GPU ({world}), no collective"}


def outg_ref_lib():
    import ctypes
    oracle = entry.load_oracle()
    if not oracle.ref_available():
        return None
    L = oracle._ref_variant(oracle.REF_PATH)
    P, I = ctypes.c_void_p, ctypes.c_int
    L.ww_outg_va.argtypes = [I, P, I, P, I, P, P, P, P, I, I] + [P] * 13 + [P, I]
    L.ww_outg_va.restype = I
    return L


def outg_call(L, igrid, c, fields, va):
    """ww_outg_va of library L on case c (synth.outg_case) into ``fields``."""
    import ctypes
    ptrs = (ctypes.c_void_p * 46)(*[f.ctypes.data for f in fields])
    a = [c[k].ctypes.data for k in ("cg", "wn", "dw", "sig", "dden", "dsii", "ecos", "esin",
                                    "ec2", "es2", "esc", "mapsf", "mapsta")]
    return L.ww_outg_va(igrid, c["ipar"].ctypes.data, 25, c["rpar"].ctypes.data, 10,
                        c["flogrd"].ctypes.data, c["flogr2"].ctypes.data, c["flogrr"].ctypes.data,
                        va.ctypes.data, va.shape[1], va.shape[0] - 1, *a, ptrs, 46)


def cpu_reference_outg(c, seconds=10.0, max_calls=20):
    L = outg_ref_lib()
    if L is None:
        return None
    import numpy as np
    va = np.array(c["va"], copy=True)
    f = [np.array(x, copy=True) for x in c["fields"]]
    if outg_call(L, 21, c, f, va) != 0:
        return None
    t0 = time.perf_counter()
    n = 0
    while True:
        outg_call(L, 21, c, f, va)
        n += 1
        el = time.perf_counter() - t0
        if el >= seconds or n >= max_calls:
            break
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return (c["nsea"] * n / el, "reference", cores,
            f"{n} W3OUTG calls on the workload's grid ({c['nsea']} sea points), OpenMP over points")


def run_b200_outg(args):
    import ctypes
    import numpy as np
    import torch
    import torch.distributed as dist

    rank, world, local = dist_env()
    if not torch.cuda.is_available():
        raise SystemExit("bench.py: no CUDA device; the B200 arm has no CPU fallback")
    torch.cuda.set_device(local)
    os.environ.setdefault("WW_KOKKOS_DEVICE_ID", str(local))
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    pkg = entry.load_package()
    synth = __import__("ww3_gpu_b200.synth", fromlist=["synth"])
    pkg.init()
    c = synth.outg_case(args.nx, args.ny, seed=2026 + rank, nk=NK, nth=NTH, ste=OUTG_STE)
    nsea, nseal = c["nsea"], int(c["ipar"][2])
    L = pkg.lib()
    P, I = ctypes.c_void_p, ctypes.c_int
    L.ww_outg_device.argtypes = [P, I, P, I, P, P, P, I, I] + [P] * 14 + [P, I, P]
    L.ww_outg_device.restype = I
    L.ww_outg_va.argtypes = [I, P, I, P, I, P, P, P, P, I, I] + [P] * 13 + [P, I]
    L.ww_outg_va.restype = I
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    handle = stream.cuda_stream

    def d(x):
        return torch.from_numpy(np.ascontiguousarray(x)).to(dev)

    names = ("cg", "wn", "dw", "sig", "dden", "dsii", "ecos", "esin", "ec2", "es2", "esc",
             "mapsf", "mapsta")
    arrs = [d(c[k]) for k in names]
    d_va = d(c["va"])
    d_f = [d(f) for f in c["fields"]]
    ebd = torch.empty(NK * nseal, dtype=torch.float32, device=dev)
    ptrs = (ctypes.c_void_p * 46)(*[t.data_ptr() for t in d_f])

    def call():
        rc = L.ww_outg_device(c["ipar"].ctypes.data, 25, c["rpar"].ctypes.data, 10,
                              c["flogrd"].ctypes.data, c["flogr2"].ctypes.data, d_va.data_ptr(),
                              c["va"].shape[1], c["va"].shape[0] - 1,
                              *[t.data_ptr() for t in arrs], ebd.data_ptr(), ptrs, 46, handle)
        if rc != 0:
            raise SystemExit(f"ww_outg_device failed ({rc})")

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if world == 1:
            return x
        tt = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        return float(tt.item())

    for _ in range(args.warmup):
        call()
    barrier()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    with ClockSampler(local) as clk:
        time.sleep(0.3)
        barrier()
        ev[0].record(stream)
        for i in range(args.steps):
            call()
            ev[i + 1].record(stream)
        barrier()
    total_ms = max_over_ranks(ev[0].elapsed_time(ev[-1]))
    per = [ev[i].elapsed_time(ev[i + 1]) for i in range(args.steps)]
    value = nsea * world * args.steps / (total_ms / 1e3)

    # ---- end to end: ww_outg_va with the VA newer on the host (it crosses every call), the
    # grid arrays copied in and the requested fields copied back
    hva = np.array(c["va"], copy=True)
    hf = [np.array(x, copy=True) for x in c["fields"]]
    ig = 1

    def host_call():
        assert L.ww_va_host_write(ig, hva.ctypes.data, hva.shape[1], hva.shape[0] - 1) == 0
        rc = outg_call(L, ig, c, hf, hva)
        if rc != 0:
            raise SystemExit(f"ww_outg_va failed ({rc})")

    host_call()
    e2e_steps = args.e2e_steps or max(3, min(args.steps, 10))
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        host_call()
    barrier()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e_value = nsea * world * e2e_steps / e2e_s
    in_bytes = int(hva.nbytes) + sum(int(c[k].nbytes) for k in names) + int(c["fields"][39].nbytes)
    out_bytes = 4 * (40 * int(c["ipar"][6]) + nseal * sum(f.shape[0] for f in c["fields"][40:]))
    peak, peak_kind = measured_peak_hbm()
    bpp = outg_bytes_per_point(c)
    call_ms = statistics.median(per)
    achieved = bpp * nsea / (call_ms / 1e3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": outg_config(args, world, c),
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": in_bytes,
                "d2h_bytes_per_step": out_bytes, "steps": e2e_steps,
                "host_entry": "ww_va_host_write + ww_outg_va"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak,
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                     "traffic": None, "kernel": "outg_init_kernel + outg_point_kernel",
                     "launch_ms": call_ms, "algorithmic_bytes_per_point": bpp},
        "gpu_launches": 2 * args.steps,
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r = cpu_reference_outg(c)
        if r is not None:
            rate, kind, cores, sample = r
            line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": cores, "kind": kind,
                                    "sample": sample}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_reference_outg(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    entry.load_package()
    synth = __import__("ww3_gpu_b200.synth", fromlist=["synth"])
    L = outg_ref_lib()
    if L is None:
        print(json.dumps({"impl": "reference", "unavailable": "the reference build "
                          "(oracle/_ref) is absent"}), flush=True)
        return 0
    import numpy as np
    c = synth.outg_case(args.nx, args.ny, seed=2026, nk=NK, nth=NTH, ste=OUTG_STE)
    va = np.array(c["va"], copy=True)
    f = [np.array(x, copy=True) for x in c["fields"]]
    for _ in range(args.warmup):
        outg_call(L, 22, c, f, va)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        outg_call(L, 22, c, f, va)
    el = time.perf_counter() - t0
    rate = c["nsea"] * args.steps / el
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    sample = f"W3OUTG calls on the workload's grid ({c['nsea']} sea points), OpenMP over points"
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": outg_config(args, 1, c),
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- the gated DIA surrogate
SUR_WORKLOAD = ("W3SNL1 36x36 on 262,144 sea points per GPU of the learned-surrogate workload's "
                "spectra (JONSWAP wind seas, 20% with a swell system, depth log-uniform 5-4000 m): "
                "the gated surrogate (BF16 MLP 1296->1024->1024->1024->1296 on tcgen05, per-point "
                "gate, rejected points on the plain DIA) against the plain DIA")
SUR_FLOP_PER_POINT = 2 * (1296 * 1024 + 2 * 1024 * 1024 + 1024 * 1296)  # 9.50e6, the model's
SUR_TRAIN_POINTS = 2_000_000
SUR_HOLDOUT = 65_536
SUR_BATCH = 8192
SUR_INFER_ROWS = 65_536


def measured_peak_bf16():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["bf16_tflops"]), "measured"
        except Exception:
            pass
    return 1590.0, "fallback"


def sur_config(args, world, train):
    return {"workload": SUR_WORKLOAD, "nk": NK, "nth": NTH, "npts_per_gpu": args.npts,
            "global_points": args.npts * world, "seed": 2024,
            "training": train,
            "hs_error": ("band-resolved Hs-tendency error per point: sum over frequency bands k "
                         "of |tau_k(S) - tau_k(S64)| / sum_k |tau_k(S64)|, tau_k = 8/Hs sum_theta "
                         "S DDEN/CG (the band's share of dHs/dt; Hs = 4 sqrt(sum A DDEN/CG) as in "
                         "the reference's W3SRCE, srce_kernel.hpp:415-430); S64 = this library's "
                         "FP64 DIA on the device; a rejected point counts its plain-DIA error; "
                         "the gate is calibrated so the mean over points is at most the budget"),
            "hs_error_budget": None,
            "l2": "inputs 1.4 GB and outputs 2.7 GB per pass > 126 MB L2 (no flush needed)",
            "parallelism": f"points sharded over {world} GPU(s), no collective; each GPU trains "
                           "its own copy of the surrogate"}


def run_reference_surrogate(args):
    """The reference has no learned part: its arm is its plain DIA (its own C++ on the host
    cores) on the same spectra, the method the gated surrogate stands in for."""
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    entry.load_package()
    synth = __import__("ww3_gpu_b200.synth", fromlist=["synth"])
    cfg, sig = synth.dia_config(NK, NTH)
    n = 2048
    g = synth.sea_states(n, seed=2024, depth_range=(5.0, 4000.0), bimodal=0.2)
    oracle = entry.load_oracle()
    if oracle.ref_available():
        run = oracle.RefSnl1(cfg, sig, igrid=1)
        kind = "reference"
        step = lambda: run(g["a"], g["cg"], g["kdmean"])  # noqa: E731
    else:
        kind = "port"
        step = lambda: oracle.w3snl1(cfg, sig, g["a"], g["cg"], g["kdmean"])  # noqa: E731
    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    el = time.perf_counter() - t0
    rate = n * args.steps / el
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    cfgd = sur_config(args, 1, "none: the reference has no learned part; this is its plain DIA")
    cfgd["reference_sample_points_per_step"] = n
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": cfgd,
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": f"{n} points of the workload's spectra per step, OpenMP over "
                                   "points (the plain DIA: the reference has no surrogate)"},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_b200_surrogate(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    rank, world, local = dist_env()
    if not torch.cuda.is_available():
        raise SystemExit("bench.py: no CUDA device; the B200 arm has no CPU fallback")
    torch.cuda.set_device(local)
    os.environ.setdefault("WW_KOKKOS_DEVICE_ID", str(local))
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    pkg = entry.load_package()
    synth = __import__("ww3_gpu_b200.synth", fromlist=["synth"])
    sur = __import__("ww3_gpu_b200.surrogate", fromlist=["surrogate"])
    cfg, sig = synth.dia_config(NK, NTH)
    grid = pkg.Snl1Grid(cfg, sig, igrid=1)
    if not args.no_autotune:  # the plain DIA kernel: every kernel that fits, timed
        pkg.snl1_autotune(1)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    handle = stream.cuda_stream

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---- set-up (untimed): training data from the plain DIA kernel, training, gate calibration
    t_setup = time.perf_counter()
    model = sur.Surrogate(1, nhidden=1024, seed=2024 + rank)
    losses = np.zeros((1, 3), np.float32)
    holdout = np.zeros(3, np.float32)
    train_s = 0.0
    if args.train_steps > 0:
        model.dataset(SUR_TRAIN_POINTS, SUR_HOLDOUT, seed=2024 + rank, bimodal=0.2, dmin=5.0,
                      dmax=4000.0)
        model.loss_weights(args.sur_mu, args.sur_lambda)
        torch.cuda.synchronize()
        t_train = time.perf_counter()
        losses = model.train(args.train_steps, batch=SUR_BATCH, lr=args.sur_lr,
                             lr_end=args.sur_lr * 0.01, seed=7 + rank)
        torch.cuda.synchronize()
        train_s = time.perf_counter() - t_train
        holdout = model.eval(SUR_TRAIN_POINTS - SUR_HOLDOUT, SUR_HOLDOUT)
    if args.gate_open:
        model.gate(1e30, 1e30)
        cal = {"open": True}
    else:
        cal = model.calibrate(65536, seed=90_001 + rank, bimodal=0.2, dmin=5.0, dmax=4000.0,
                              energy=args.sur_energy, target=args.sur_target)
    setup_s = time.perf_counter() - t_setup

    npts = args.npts
    a = torch.empty(npts, NK * NTH, device=dev)
    cg = torch.empty(npts, NK, device=dev)
    kd = torch.empty(npts, device=dev)
    model.synth(npts, a, cg, kd, seed=31_337 + rank, bimodal=0.2, dmin=5.0, dmax=4000.0)
    s = torch.empty_like(a)
    d = torch.empty_like(a)
    s_plain = torch.empty_like(a)
    d_plain = torch.empty_like(a)
    barrier()

    def timed(fn, steps, warmup, ev_per_step=False):
        for _ in range(warmup):
            fn()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        barrier()
        return max_over_ranks(e0.elapsed_time(e1))

    # ---- the plain DIA (the method without the learned part), same points, same clock
    plain_ms = timed(lambda: grid.run_device(npts, a, cg, kd, s_plain, d_plain, handle),
                     args.steps, args.warmup) / args.steps
    # ---- the gated surrogate: value
    with ClockSampler(local) as clk:
        time.sleep(0.3)
        total_ms = timed(lambda: model.gated(npts, a, cg, kd, s, d, None, handle), args.steps,
                         args.warmup)
    gated_ms = total_ms / args.steps
    value = npts * world * args.steps / (total_ms / 1e3)
    fallback = model.fallback_count(handle)

    # ---- every result's error against the FP64 DIA (this library's, on the device)
    stats = torch.empty(npts, 10, dtype=torch.float64, device=dev)
    model.judge(npts, a, cg, kd, s, stats, stream=handle)
    err_gated = sur.error_summary(stats.cpu().numpy())
    model.judge(npts, a, cg, kd, s_plain, stats, stream=handle)
    err_plain = sur.error_summary(stats.cpu().numpy())

    # ---- the network alone (the four tcgen05 GEMMs), for the roofline
    rows = SUR_INFER_ROWS
    x = torch.randn(rows, 1344, device=dev).to(torch.bfloat16)
    out = torch.empty(rows, 1344, device=dev)
    fwd_ms = timed(lambda: model.forward(rows, x, out, handle), 20, 3) / 20
    achieved = SUR_FLOP_PER_POINT * rows / (fwd_ms / 1e3) / 1e12
    peak, peak_kind = measured_peak_bf16()

    # ---- end to end: page-locked host inputs in, S and D out, every step
    e2e_steps = args.e2e_steps or max(3, min(args.steps, 5))
    h_a, h_cg, h_kd = a.cpu().pin_memory(), cg.cpu().pin_memory(), kd.cpu().pin_memory()
    h_s = torch.empty_like(h_a).pin_memory()
    h_d = torch.empty_like(h_a).pin_memory()

    def e2e_step():
        model.gated_host(npts, h_a, h_cg, h_kd, h_s, h_d)

    e2e_step()
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    barrier()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e_value = npts * world * e2e_steps / e2e_s
    same = bool(torch.equal(h_s.view(torch.int32), s.cpu().view(torch.int32)))

    chunks = (npts + SUR_INFER_ROWS - 1) // SUR_INFER_ROWS
    train = {"points": SUR_TRAIN_POINTS, "holdout": SUR_HOLDOUT, "steps": args.train_steps,
             "batch": SUR_BATCH, "lr": args.sur_lr, "mu": args.sur_mu, "lambda": args.sur_lambda,
             "train_s": train_s, "ms_per_step": 1e3 * train_s / max(1, args.train_steps),
             "setup_s": setup_s, "loss_first": [float(v) for v in losses[:50].mean(axis=0)],
             "loss_last": [float(v) for v in losses[-200:].mean(axis=0)],
             "holdout_loss": [float(v) for v in holdout], "gate": cal,
             "train_tflops": (3 * SUR_FLOP_PER_POINT * SUR_BATCH * args.train_steps
                              / max(train_s, 1e-9) / 1e12)}
    cfgd = sur_config(args, world, train)
    cfgd["hs_error_budget"] = args.sur_target
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": gated_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "bf16 network / f32 fallback",
        "data": "synthetic", "config": cfgd,
        "plain_dia": {"value": npts * world / (plain_ms / 1e3), "unit": UNIT,
                      "ms_per_step": plain_ms, "kernel": "snl1_pairtile_kernel (the default DIA)",
                      "error_vs_fp64": err_plain},
        "speedup_vs_plain": plain_ms / gated_ms,
        "accepted_fraction": 1.0 - fallback / npts,
        "error_vs_fp64": err_gated,
        "e2e": {"value": e2e_value, "unit": UNIT,
                "h2d_bytes_per_step": int((h_a.numel() + h_cg.numel() + h_kd.numel()) * 4),
                # S whole; of D only each chunk's packed rejected rows (8,192-row slot, its
                # index list and count): the accepted points' D is zero and the entry clears it
                # on the host while the device works (a chunk rejecting more than 8,192 points
                # would bring its whole D; none did when this line was measured)
                "d2h_bytes_per_step": int(h_s.numel() * 4 + chunks * (4 + 8192 * 4 +
                                                                      8192 * 1296 * 4)),
                "steps": e2e_steps, "host_entry": "ww_snl1_gated_host (page-locked host buffers; copies "
                                                  "pipelined with the compute in 65,536-point chunks; "
                                                  "D cleared on the host, rejected rows copied back)",
                "matches_device_entry": same},
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak,
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json bf16_tflops, burst)",
                     "traffic": None, "kernel": "gemm_kernel (tcgen05, 4 launches per forward)",
                     "forward_ms_65536_rows": fwd_ms,
                     "algorithmic_flop_per_point": SUR_FLOP_PER_POINT},
        "gpu_launches": args.steps * chunks * 7,
        "autotune": pkg.autotune_report(),
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        g = {"a": a[:4096].cpu().numpy(), "cg": cg[:4096].cpu().numpy(),
             "kdmean": kd[:4096].cpu().numpy()}
        rate, kind, cores, sample = cpu_reference_rate(cfg, sig, g)
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": cores, "kind": kind,
                                "sample": sample + " (the plain DIA: the reference has no "
                                                   "surrogate)"}
    if rank == 0 and world == 1 and not args.no_srce_line:
        line["w3srce_config1"] = run_b200_srce(args, quiet=True, npts=SRCE_NPTS, steps=10, igrid=2,
                                               warmup=3)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.workload == "surrogate":
        return (run_reference_surrogate(args) if args.impl == "reference"
                else run_b200_surrogate(args))
    if args.workload == "dia":
        return run_reference_dia(args) if args.impl == "reference" else run_b200_dia(args)
    if args.workload == "step":
        return run_reference_step(args) if args.impl == "reference" else run_b200_step(args)
    if args.workload == "outg":
        return run_reference_outg(args) if args.impl == "reference" else run_b200_outg(args)
    if args.workload == "multigrid":
        return (run_reference_multigrid(args) if args.impl == "reference"
                else run_b200_multigrid(args))
    return run_reference_srce(args) if args.impl == "reference" else run_b200_srce(args)


if __name__ == "__main__":
    sys.exit(main())
