"""The plain form's FP64 special functions on the device (set_b200/csrc/mhd_core.cuh: rs_rcp,
rs_rsqrt, rs_sqrt: Newton-refined approximate instructions) against IEEE results; its quotient
from a shared correctly rounded reciprocal (div_rn) against IEEE division; and its exact primitive
recovery (prim_from_cons<true>) against the oracle's, bit for bit.

tests/csrc/rs_special.cu wraps them in a kernel; this test compiles it with nvcc for sm_100a
into a temporary library.  The reference values are numpy's correctly rounded 1/x and sqrt(x),
and 1/sqrt(x) evaluated in extended precision and rounded once.
"""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "set_b200", "csrc")


@pytest.fixture(scope="module")
def rs_lib(tmp_path_factory):
    nvcc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    nvcc = nvcc if os.path.exists(nvcc) else shutil.which("nvcc")
    out = str(tmp_path_factory.mktemp("rs") / "librs.so")
    subprocess.check_call([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
                           "-Xcompiler", "-fPIC", "-shared", "-I" + CSRC,
                           os.path.join(HERE, "csrc", "rs_special.cu"), "-o", out])
    lib = C.CDLL(out)
    dp = C.POINTER(C.c_double)
    lib.rs_eval.restype = C.c_int
    lib.rs_eval.argtypes = [dp, dp, C.c_longlong]
    lib.div_eval.restype = C.c_int
    lib.div_eval.argtypes = [dp, dp, dp, C.c_longlong]
    lib.prim_eval.restype = C.c_int
    lib.prim_eval.argtypes = [dp, dp, C.c_longlong]
    return lib


def rs_eval(lib, x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.zeros((x.size, 3))
    rc = lib.rs_eval(x.ctypes.data_as(C.POINTER(C.c_double)), out.ctypes.data_as(C.POINTER(C.c_double)), x.size)
    assert rc == 0
    return out


def ulps(a, b):
    """Distance in units in the last place between doubles of the same sign."""
    ia = a.view(np.int64)
    ib = b.view(np.int64)
    return np.abs(ia - ib)


def test_special_functions_on_their_domain(rs_lib):
    rng = np.random.default_rng(1)
    x = 10.0 ** rng.uniform(-300.0, 300.0, 1 << 20)
    r = rs_eval(rs_lib, x)
    rcp_ref = 1.0 / x
    sqrt_ref = np.sqrt(x)
    rsq_ref = (np.longdouble(1.0) / np.sqrt(x.astype(np.longdouble))).astype(np.float64)
    d_rcp, d_rsq, d_sqrt = ulps(r[:, 0], rcp_ref), ulps(r[:, 1], rsq_ref), ulps(r[:, 2], sqrt_ref)
    assert d_rcp.max() <= 1 and d_rsq.max() <= 1 and d_sqrt.max() <= 2, (d_rcp.max(), d_rsq.max(), d_sqrt.max())
    # 1/x and 1/sqrt(x) within one ulp, sqrt(x) = x (1/sqrt(x)) within two, most correctly rounded
    cr = [(d == 0).mean() for d in (d_rcp, d_rsq, d_sqrt)]
    print("correctly rounded fraction (1/x, 1/sqrt(x), sqrt(x)):", cr)
    assert min(cr) >= 0.6, cr
    # negative arguments of the reciprocal (SL - SM < 0 in the flux)
    rn = rs_eval(rs_lib, -x[:4096])
    assert ulps(-rn[:, 0], rcp_ref[:4096]).max() <= 1


def test_special_functions_outside_their_domain(rs_lib):
    """The documented edge behaviour: sqrt(0) = 0; 1/x is NaN at 0, inf and subnormals, 1/sqrt(x)
    is NaN at 0 and inf and +inf at subnormals (the approximate instructions flush subnormals).
    The flux never passes them such arguments from a valid state."""
    edge = np.array([0.0, np.inf, 5e-324, 1e-310])
    r = rs_eval(rs_lib, edge)
    assert r[0, 2] == 0.0
    assert np.isnan(r[:, 0]).all() and np.isnan(r[:2, 1]).all() and (r[2:, 1] == np.inf).all()


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def test_quotient_from_shared_reciprocal_is_ieee_division(rs_lib):
    """div_rn(a, b, RN(1/b)) equals the device's IEEE a / b bit for bit: quotients over 1e-150..1e150
    of both signs, and the state's own range (velocities of momenta over densities)."""
    rng = np.random.default_rng(2)
    n = 1 << 20
    a = np.concatenate([rng.choice([-1.0, 1.0], n) * 10.0 ** rng.uniform(-150, 150, n),
                        rng.normal(0.0, 500.0, n)])
    b = np.concatenate([rng.choice([-1.0, 1.0], n) * 10.0 ** rng.uniform(-150, 150, n),
                        10.0 ** rng.uniform(-4, 4, n)])
    a[:7] = [0.0, -0.0, 1.0, 3.0, 7.0, 1.0, 0.1]
    b[:7] = [3.0, 5.0, 3.0, 3.0, 3.0, 1.0 - 2.0 ** -53, 3.5449077018110318]
    out = np.zeros(2 * a.size)
    assert rs_lib.div_eval(_p(a), _p(b), _p(out), a.size) == 0
    got, ieee = out[0::2], out[1::2]
    np.testing.assert_array_equal(got.view(np.int64), ieee.view(np.int64))
    np.testing.assert_array_equal(ieee, a / b)   # the device's division is numpy's


def test_exact_primitive_recovery_matches_the_oracle(rs_lib):
    """prim_from_cons<true> on the device equals the oracle's prim_from_cons bit for bit,
    including hypersonic states whose pressure is ~1e-4 of the kinetic energy (where one ulp of
    a velocity moves p by ~1e-12)."""
    import oracle as O
    rng = np.random.default_rng(3)
    n = 1 << 16
    rho = 10.0 ** rng.uniform(-3, 2, n)
    v = rng.normal(0.0, 3.0, (n, 3)) * np.where(rng.uniform(size=n) < 0.3, 5.0, 1.0)[:, None]
    B = rng.normal(0.0, 1.0, (n, 3)) * (rng.uniform(size=n) < 0.7)[:, None]
    ke = 0.5 * rho * (v ** 2).sum(1)
    me = 0.5 * (B ** 2).sum(1) / (4 * np.pi)
    p = (ke + me) * 10.0 ** rng.uniform(-4, 1, n)
    U = np.zeros((n, 8))
    U[:, 0] = rho
    U[:, 1:4] = rho[:, None] * v
    U[:, 4] = p / (2.0 / 3.0) + ke + me
    U[:, 5:8] = B
    got = np.zeros((n, 8))
    assert rs_lib.prim_eval(_p(U), _p(got), n) == 0
    ref = np.array([O.prim_from_cons(U[i]) for i in range(n)])
    np.testing.assert_array_equal(got.view(np.int64), ref.view(np.int64))
