"""Throughput of the B200 instructions the stage kernels' costs are made of (tests/csrc/pipe_rates.cu),
in thread operations per SM clock: FP64 fused multiply-add, an FP64 -> FP32 -> FP64 conversion pair
(with one FP64 multiply), FP32 fused multiply-add, the FP64 reciprocal seed (with one FP64 add), and
the library fmin / fmax of doubles (with one FP64 add).  These are the figures behind the design
notes on the plain and mixed forms: FP64 runs at half the FP32 rate, a conversion between the two
costs several FP64 operations, and the library min / max of doubles is a long sequence (the
kernels use compare-and-select or integer forms instead).  Run with -s to print the table.
"""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
NAMES = ["DFMA", "F2F pair + DMUL", "FFMA", "MUFU rcp64 + DADD", "fmin + fmax + DADD"]


def test_pipe_rates(tmp_path):
    nvcc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    nvcc = nvcc if os.path.exists(nvcc) else shutil.which("nvcc")
    lib_path = str(tmp_path / "libpipe.so")
    subprocess.check_call([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-Xcompiler", "-fPIC",
                           "-shared", os.path.join(HERE, "csrc", "pipe_rates.cu"), "-o", lib_path])
    lib = C.CDLL(lib_path)
    lib.pipe_rates.restype = C.c_int
    lib.pipe_rates.argtypes = [C.POINTER(C.c_double)]
    r = np.zeros(5)
    assert lib.pipe_rates(r.ctypes.data_as(C.POINTER(C.c_double))) == 0
    for name, v in zip(NAMES, r):
        print(f"{name:22s} {v:8.2f} per SM clock")
    # FP64 is a half-rate pipe and FP32 a full-rate one (64 and 128 lanes per SM clock); the
    # conversion pair and the library min / max are far slower than one FP64 operation
    assert 40.0 < r[0] < 70.0 and r[2] > 1.5 * r[0]
    assert r[1] < 0.5 * r[0] and r[4] < 0.5 * r[0]
