"""Shared fixtures. Tests marked ``gpu`` need a CUDA device and run the library's kernels
through its C ABI; everything else runs on the CPU (oracle pins, host logic, library loading)."""

import pathlib
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

import __graft_entry__ as entry  # noqa: E402

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def cuda_available():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def pkg():
    return entry.load_package()


@pytest.fixture(scope="session")
def oracle():
    o = entry.load_oracle()
    o.lib()
    return o


@pytest.fixture(scope="session")
def synth(pkg):
    import importlib

    return importlib.import_module("ww3_gpu_b200.synth")


@pytest.fixture(scope="session")
def golden():
    g = dict(np.load(GOLDEN / "snl1_nk25_nth24.npz"))
    cfg = {k: (int(g[k]) if k in ("nk", "nth") else float(g[k]))
           for k in ("nk", "nth", "xfr", "dth", "lam", "snlc1", "kdcon", "kdmn", "snls1",
                     "snls2", "snls3", "fachfe")}
    g["cfg"] = cfg
    return g


def bits(x):
    return np.ascontiguousarray(x, np.float32).view(np.uint32)


def assert_bitexact(x, y, what=""):
    bx, by = bits(x), bits(y)
    if not np.array_equal(bx, by):
        n = int(np.sum(bx != by))
        diff = np.abs(np.asarray(x, np.float64) - np.asarray(y, np.float64))
        raise AssertionError(f"{what}: {n} of {bx.size} values differ (max abs diff {diff.max():.3e})")
