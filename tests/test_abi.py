"""The C ABI of libww_b200.so without a GPU: it loads, exports every declared symbol, resolves
the run-time flags as the reference's part_flags.cpp does, validates before it computes, and
refuses to run (loudly, with a status) when there is no CUDA device."""

import os
import pathlib
import re
import subprocess
import sys
import textwrap

import pytest

from conftest import ROOT, cuda_available

HEADER = ROOT / "include" / "ww_b200.h"


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(ww_[a-z0-9_]+)\s*\(", text)))


def test_header_declarations_are_the_package_list(pkg):
    assert declared_functions() == sorted(pkg.EXPORTS)


def test_library_exports_every_declared_symbol(pkg):
    out = subprocess.run(["nm", "-D", "--defined-only", str(pkg.LIB_PATH)], check=True,
                         capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    missing = [f for f in declared_functions() if f not in exported]
    assert not missing, missing
    L = pkg.lib()
    for f in declared_functions():
        assert hasattr(L, f)


def test_library_is_built_for_sm100a_only():
    """Every CUDA source is compiled with the one sm_100a target of the Makefile (the library
    then runs on a B200 or not at all: the GPU tests are the run-time half of this check)."""
    mk = (ROOT / "ww3-gpu_b200" / "csrc" / "Makefile").read_text()
    arch = re.search(r"^ARCH := (.*)$", mk, flags=re.M).group(1).strip()
    assert arch == "-gencode arch=compute_100a,code=sm_100a"
    flag_sets = re.findall(r"^(\w+FLAGS) := \$\(ARCH\)", mk, flags=re.M)
    assert set(flag_sets) == {"NVFLAGS", "MLPFLAGS"}
    nvcc_lines = [ln for ln in mk.splitlines() if ln.strip().startswith("$(NVCC)")]
    assert nvcc_lines and all("$(ARCH)" in ln or "FLAGS)" in ln for ln in nvcc_lines)


def run_py(code, env=None):
    e = dict(os.environ)
    for k in list(e):
        if k.startswith("WW_KOKKOS_"):
            del e[k]
    e.update(env or {})
    r = subprocess.run([sys.executable, "-c", textwrap.dedent(code)], env=e, cwd=str(ROOT),
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    return r.stdout.strip()


FLAG_CODE = """
import __graft_entry__ as g
p = g.load_package()
L = p.lib()
names = ["WW_KOKKOS_SNL1", "WW_KOKKOS_SRCE", "WW_KOKKOS_XYP3", "WW_KOKKOS_KTP3", "WW_KOKKOS_SDS4"]
print(" ".join(str(L.ww_kokkos_flag(n.encode())) for n in names), L.ww_kokkos_preset_status(),
      L.ww_kokkos_strict(), L.ww_snl1_enabled())
"""


@pytest.mark.parametrize("env,expect", [
    ({}, "0 0 0 0 0 0 0 0"),
    ({"WW_KOKKOS_SNL1": "1"}, "1 0 0 0 0 0 0 1"),
    ({"WW_KOKKOS_SNL1": "yes"}, "0 0 0 0 0 0 0 0"),
    ({"WW_KOKKOS_ALL": "1"}, "2 2 0 0 2 0 0 1"),           # XYP3/KTP3 are opt-in only
    ({"WW_KOKKOS_ALL": "1", "WW_KOKKOS_SRCE": "0"}, "2 0 0 0 2 0 0 1"),
    ({"WW_KOKKOS_PRESET": "resident"}, "0 1 1 1 0 1 0 0"),
    ({"WW_KOKKOS_PRESET": "nope"}, "0 0 0 0 0 -1 0 0"),
    ({"WW_KOKKOS_STRICT": "1"}, "0 0 0 0 0 0 1 0"),
])
def test_run_time_flags(env, expect):
    assert run_py(FLAG_CODE, env) == expect


def test_fallback_slots():
    out = run_py("""
    import __graft_entry__ as g
    L = g.load_package().lib()
    a = L.ww_kokkos_fallback_slot(b"SRCE"); b = L.ww_kokkos_fallback_slot(b"XYP3")
    c = L.ww_kokkos_fallback_slot(b"SRCE"); d = L.ww_kokkos_fallback_slot(b"X" * 40)
    L.ww_kokkos_fallback_add(a); L.ww_kokkos_fallback_add(a); L.ww_kokkos_fallback_add(99)
    print(a, b, c, d)
    """)
    assert out == "0 1 0 -1"


def test_compute_before_init_is_not_initialised(pkg):
    import numpy as np

    L = pkg.lib()
    a = np.zeros((2, 1296), np.float32)
    s = np.full_like(a, 7.0)
    L.ww_snl1(123, 2, a.ctypes.data, a.ctypes.data, a.ctypes.data, s.ctypes.data, s.ctypes.data)
    assert L.ww_snl1_last_error() == pkg.ERR_NOT_INITIALISED
    assert np.all(s == 7.0)  # nothing written on a validation failure
    L.ww_snl1_device(123, 2, 0, 0, 0, 0, 0, None)
    assert L.ww_snl1_last_error() == pkg.ERR_NOT_INITIALISED
    assert L.ww_snl1_select_kernel(123, 0) == -1


@pytest.mark.skipif(cuda_available(), reason="checks the no-device path")
def test_init_without_device_fails_loudly(pkg):
    out = run_py("""
    import __graft_entry__ as g
    p = g.load_package()
    rc = p.lib().ww_kokkos_init(-1)
    try:
        p.Snl1Grid({"nk": 36, "nth": 36, "xfr": 1.1, "dth": 0.17, "lam": 0.25, "snlc1": 1.0,
                    "kdcon": 0.75, "kdmn": 0.5, "snls1": 5.5, "snls2": 0.833, "snls3": -1.25,
                    "fachfe": 0.62}, [0.2] * 36)
        print(rc, "no-error")
    except RuntimeError as e:
        print(rc, "raised")
    """)
    assert out == "4 raised"
