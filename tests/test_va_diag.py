"""The resident VA's diagnostics, each in a child process since the flags are read once per
process (the reference's resident_c.hpp:18-37 and its mutation audit): WW_KOKKOS_VA_POISON fills
the host VA with a quiet NaN whenever the device copy becomes the newer one, so a host read that
skipped its ww_va_host_read shows; WW_KOKKOS_VA_CHECK catches a host VA changed behind the state's
back; WW_KOKKOS_VA_COUNT prints the copy counts at exit."""

import os
import pathlib
import subprocess
import sys

import pytest

from conftest import cuda_available

ROOT = pathlib.Path(__file__).resolve().parents[1]
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

CHILD = r'''
import sys
import numpy as np
sys.path.insert(0, ROOT)
import __graft_entry__ as e
pkg = e.load_package()
synth = __import__("ww3_gpu_b200.synth", fromlist=["synth"])
case = synth.ktp3_case(64, seed=3, nsea=64)
va = np.array(case["va"], np.float32, copy=True)
ref = np.array(case["va"], np.float32, copy=True)
rc, out, _, _ = pkg.ktp3_batch(case)            # the same call on the host-pointer entry
assert rc == 0
rc, _, _, _ = pkg.ktp3_batch(case, igrid=5, va=va)   # resident: the device copy is now newer
print("rc1", rc)
print("poisoned", int(np.all(va.view(np.uint32) == 0x7FC0FA11)))
pkg.va_host_read(5, va)
print("restored", int(np.array_equal(va.view(np.uint32), out.view(np.uint32))))
va[1, 0] += 1.0                                  # a host change that no ww_va_host_write declares
rc, _, _, _ = pkg.ktp3_batch(case, igrid=5, va=va)
print("rc2", rc)
'''


def run_child(env_flag):
    env = dict(os.environ)
    env[env_flag] = "1"
    code = CHILD.replace("ROOT", repr(str(ROOT)))
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env,
                       cwd=str(ROOT), timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    vals = dict(line.split() for line in p.stdout.splitlines() if line.split()[:1] and
                line.split()[0] in ("rc1", "poisoned", "restored", "rc2"))
    return vals, p.stderr


def test_poison():
    vals, err = run_child("WW_KOKKOS_VA_POISON")
    assert vals["rc1"] == "0" and vals["poisoned"] == "1" and vals["restored"] == "1", (vals, err)


def test_check_catches_an_undeclared_host_write():
    vals, err = run_child("WW_KOKKOS_VA_CHECK")
    assert vals["rc1"] == "0" and vals["poisoned"] == "0" and vals["restored"] == "1", (vals, err)
    assert vals["rc2"] != "0", (vals, err)
    assert "WW_KOKKOS_VA_CHECK" in err and "changed since the last sync" in err, err


def test_count_report():
    vals, err = run_child("WW_KOKKOS_VA_COUNT")
    assert vals["rc1"] == "0" and vals["rc2"] == "0", (vals, err)
    assert "[va] traffic:" in err and "whole uploads" in err and "whole downloads" in err, err
