"""The DEVICE build of ww3-gpu_b200/csrc/libm_dev.cuh on a B200 against this host's glibc: every
float input of the unary functions (all 2^32 bit patterns) and 2^28 seeded argument pairs of powf
and atan2f (tests/libm_device_check.cu). test_libm.py checks the host build of the same source;
this checks the bits the kernels actually compute. NaN results compare equal whatever their
payload."""

import pathlib
import re
import subprocess

import pytest

from conftest import cuda_available

ROOT = pathlib.Path(__file__).resolve().parents[1]
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    exe = tmp_path_factory.mktemp("libm_dev") / "libm_device_check"
    subprocess.run(["/usr/local/cuda/bin/nvcc", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-O3", "-std=c++17", "-fmad=false", "-prec-div=true", "-prec-sqrt=true",
                    "-ftz=false", "-Xcompiler", "-fopenmp", "-Xcompiler", "-ffp-contract=off",
                    "-ccbin", "/usr/bin/g++", str(ROOT / "tests" / "libm_device_check.cu"),
                    "-o", str(exe), "-lgomp"], check=True)
    return exe


@pytest.mark.parametrize("fn,stride", [("expf", 1), ("logf", 1), ("sinf", 1), ("cosf", 1),
                                       ("tanhf", 1), ("atanf", 1), ("log10f", 1), ("sinhf", 1),
                                       ("coshf", 1), ("powf", 16), ("atan2f", 16)])
def test_device_libm_equals_glibc(checker, fn, stride):
    out = subprocess.run([str(checker), fn, str(stride)], check=True, capture_output=True,
                         text=True).stdout
    m = re.search(r"checked (\d+) mismatches (\d+) first (-?\d+)", out)
    assert m, out
    assert int(m.group(1)) == (1 << 32) // stride
    assert int(m.group(2)) == 0, out
