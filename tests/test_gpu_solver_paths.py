"""The region-first solver paths against the branch-free ones, on the device.

The FP64 / FP32 HLLD and HLLC solvers (set_b200/csrc/mhd_core.cuh, riemann<..., LAZY>) find the
wave-fan region first and skip the quantities the selected region does not read (an FR face,
SR < 0, needs no star state); the delta form's solver (riemann_delta<..., LAZY>) converts only
what the wave speeds need on FR faces.  The formulas are the same, so the results must agree
with the branch-free evaluation's to rounding; they are not bit for bit the same, because the
compiler fuses a multiply into an add (FMA) where the product has one use in its basic block,
and the two forms place the same expressions in different blocks.  Measured on a B200: HLLD
fluxes within ~2e-14 of the face's largest flux component (~98 % of faces bit for bit), HLLC
within ~2e-13 (~1/3 bit for bit); the delta form to its FP32 corrections' rounding.  The
pressure floor's quick test (pressure_surely_positive) must never clear a state whose exact
recovery gives p <= 0, and the guarded primitive recovery (prim_from_cons_guarded) must be the
exact one where it matters and within stated bounds elsewhere.

tests/csrc/solver_paths.cu wraps the instantiations in kernels; this test compiles it with nvcc
for sm_100a into a temporary library.
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
GAMMA = 5.0 / 3.0
SPI4 = np.sqrt(4.0 * np.pi)


@pytest.fixture(scope="module")
def sp_lib(tmp_path_factory):
    nvcc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    nvcc = nvcc if os.path.exists(nvcc) else shutil.which("nvcc")
    out = str(tmp_path_factory.mktemp("sp") / "libsp.so")
    subprocess.check_call([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
                           "-Xcompiler", "-fPIC", "-shared", "-I" + CSRC,
                           os.path.join(HERE, "csrc", "solver_paths.cu"), "-o", out])
    lib = C.CDLL(out)
    dp = C.POINTER(C.c_double)
    lib.riemann_pair.restype = C.c_int
    lib.riemann_pair.argtypes = [dp, dp, C.c_longlong, C.c_int, C.c_int, C.c_int, dp, dp]
    lib.delta_pair.restype = C.c_int
    lib.delta_pair.argtypes = [dp, dp, C.c_longlong, C.c_int, dp, dp]
    lib.pressure_test.restype = C.c_int
    lib.pressure_test.argtypes = [dp, C.c_longlong, C.POINTER(C.c_int)]
    lib.guarded_recovery.restype = C.c_int
    lib.guarded_recovery.argtypes = [dp, C.c_longlong, dp]
    return lib


def _ptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def face_states(n, seed, field=True):
    """Face-frame primitive pairs over every wave-fan region: supersonic either way (FR, FL),
    subsonic with both signs of the contact speed, near-zero normal field, small and large jumps."""
    rng = np.random.default_rng(seed)
    q1 = np.empty((n, 8))
    q1[:, 0] = 10.0 ** rng.uniform(-2, 1, n)
    q1[:, 1] = rng.uniform(-15, 15, n)
    q1[:, 2:4] = rng.uniform(-3, 3, (n, 2))
    q1[:, 4] = 10.0 ** rng.uniform(-3, 1, n)
    q1[:, 5:8] = rng.uniform(-3, 3, (n, 3)) if field else 0.0
    if field:
        q1[rng.random(n) < 0.15, 5] = 0.0
    near = rng.random(n) < 0.5
    q2 = np.where(near[:, None], q1 * (1.0 + rng.uniform(-0.05, 0.05, (n, 8))), np.empty((n, 8)))
    far = ~near
    m = int(far.sum())
    q2[far, 0] = 10.0 ** rng.uniform(-2, 1, m)
    q2[far, 1] = rng.uniform(-15, 15, m)
    q2[far, 2:4] = rng.uniform(-3, 3, (m, 2))
    q2[far, 4] = 10.0 ** rng.uniform(-3, 1, m)
    q2[far, 5:8] = rng.uniform(-3, 3, (m, 3)) if field else 0.0
    q2[:, 5] = np.where(rng.random(n) < 0.7, q1[:, 5], q2[:, 5])   # mostly a continuous normal field
    return np.ascontiguousarray(q1), np.ascontiguousarray(q2)


def _bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.int64), np.ascontiguousarray(b).view(np.int64))


def _agree(lazy, eager, tol, stol):
    """Speeds (SL, SR, SM) within stol of max(|SL|, |SR|); flags equal on all but faces at a
    region boundary; fluxes within tol of the face's largest flux component.  Returns the largest
    flux deviation and the fraction of faces equal bit for bit."""
    S_l, S_e = lazy[:, 8:11], eager[:, 8:11]
    assert np.array_equal(np.isnan(S_l), np.isnan(S_e))
    sscale = np.abs(S_e[:, :2]).max(1, keepdims=True) + 1e-300
    sdev = float(np.nanmax(np.abs(S_l - S_e) / sscale))
    assert sdev <= stol, sdev
    same_flag = lazy[:, 11] == eager[:, 11]
    assert same_flag.mean() >= 0.9999, same_flag.mean()
    Fl, Fe = lazy[same_flag, :8], eager[same_flag, :8]
    assert np.array_equal(np.isnan(Fl), np.isnan(Fe))
    ok = np.isfinite(Fe).all(1)
    scale = np.abs(Fe[ok]).max(1, keepdims=True) + 1e-300
    dev = float((np.abs(Fl[ok] - Fe[ok]) / scale).max())
    same = float((lazy.view(np.int64) == eager.view(np.int64)).all(1).mean())
    assert dev <= tol, (dev, same)
    return dev, same


def _regions_covered(out):
    SL, SR = out[:, 8], out[:, 9]
    fr, fl = SR < 0, SL > 0
    star = ~fr & ~fl
    assert fr.mean() > 0.05 and fl.mean() > 0.05 and star.mean() > 0.2, (fr.mean(), fl.mean(), star.mean())


@pytest.mark.parametrize("nstate", [2, 3])
@pytest.mark.parametrize("mode,n_disc", [(0, 0), (1, 0), (2, 0), (0, 1), (0, 2), (2, 1)])
def test_region_first_solver_is_the_branch_free_one(sp_lib, nstate, mode, n_disc):
    n = 1 << 18
    q1, q2 = face_states(n, seed=11 + 7 * nstate + mode + 3 * n_disc)
    lazy = np.zeros((n, 12))
    eager = np.zeros((n, 12))
    rc = sp_lib.riemann_pair(_ptr(q1), _ptr(q2), n, nstate, n_disc, mode, _ptr(lazy), _ptr(eager))
    assert rc == 0
    _regions_covered(eager)
    dev, same = _agree(lazy, eager, 1e-4 if mode == 2 else 1e-12, 1e-5 if mode == 2 else 1e-13)
    print(f"riemann nstate={nstate} mode={mode} n_disc={n_disc}: max deviation {dev:.2e}, bitwise equal {same:.3f}")


@pytest.mark.parametrize("nstate", [2, 3])
def test_delta_form_fr_path_is_the_full_path(sp_lib, nstate):
    n = 1 << 18
    q1, q2 = face_states(n, seed=40 + nstate, field=(nstate == 3))
    lazy = np.zeros((n, 12))
    eager = np.zeros((n, 12))
    rc = sp_lib.delta_pair(_ptr(q1), _ptr(q2), n, nstate, _ptr(lazy), _ptr(eager))
    assert rc == 0
    _regions_covered(eager)
    # the delta form's star corrections are FP32: a one-rounding difference upstream moves them by
    # FP32 rounding of the side fluxes, which is large against the final flux where the two cancel
    dev, same = _agree(lazy, eager, 1e-4, 1e-5)
    print(f"delta nstate={nstate}: max deviation {dev:.2e}, bitwise equal {same:.3f}")


def test_quick_pressure_test_never_clears_a_floored_state(sp_lib):
    rng = np.random.default_rng(5)
    n = 1 << 20
    U = np.empty((n, 8))
    rho = 10.0 ** rng.uniform(-3, 2, n)
    U[:, 0] = rho
    U[:, 1:4] = rng.uniform(-1, 1, (n, 3)) * rho[:, None] * (10.0 ** rng.uniform(-2, 2, n))[:, None]
    U[:, 5:8] = rng.uniform(-3, 3, (n, 3)) * (rng.random(n) < 0.8)[:, None]
    ke = 0.5 * (U[:, 1:4] ** 2).sum(1) / rho
    me = 0.5 * (U[:, 5:8] ** 2).sum(1) / (4.0 * np.pi)
    # half the states a few tens of ulps either side of p = 0, half with p well above it
    edge = rng.random(n) < 0.5
    rel = np.where(edge, rng.uniform(-64, 64, n) * 2.0 ** -52, 10.0 ** rng.uniform(-3, 0, n))
    U[:, 4] = (ke + me) * (1.0 + rel)
    out = np.zeros(2 * n, dtype=np.int32)
    rc = sp_lib.pressure_test(_ptr(np.ascontiguousarray(U)), n, out.ctypes.data_as(C.POINTER(C.c_int)))
    assert rc == 0
    quick, exact = out[0::2].astype(bool), out[1::2].astype(bool)
    assert not np.any(quick & ~exact), np.argwhere(quick & ~exact)[:5]
    # the quick test clears nearly every state away from the floor; the edge set holds floored ones
    assert quick[~edge].mean() > 0.999
    assert (~exact[edge]).sum() > 1000


def test_guarded_recovery_is_the_exact_one_where_it_matters(sp_lib):
    """prim_from_cons_guarded: the exact recovery bit for bit wherever ke + me > 64 p (the
    hypersonic source outflow); elsewhere each velocity is the product with a one-ulp reciprocal,
    within 4 ulps of the correctly rounded quotient, and p within 1e-13 relative (about
    12 (ke + me) / p + 2 E / p ulps, at most ~8.5e-14 under the guard)."""
    rng = np.random.default_rng(9)
    n = 1 << 20
    rho = 10.0 ** rng.uniform(-3, 2, n)
    vel = rng.uniform(-1, 1, (n, 3)) * (10.0 ** rng.uniform(-2, 2, n))[:, None]
    B = rng.uniform(-3, 3, (n, 3)) * (rng.random(n) < 0.8)[:, None]
    p = 10.0 ** rng.uniform(-4, 1, n)
    U = np.empty((n, 8))
    U[:, 0] = rho
    U[:, 1:4] = rho[:, None] * vel
    U[:, 5:8] = B
    ke = 0.5 * rho * (vel ** 2).sum(1)
    me = 0.5 * (B ** 2).sum(1) / (4.0 * np.pi)
    U[:, 4] = p * 1.5 + ke + me
    out = np.zeros((n, 16))
    assert sp_lib.guarded_recovery(_ptr(U), n, _ptr(out)) == 0
    g, x = out[:, :8], out[:, 8:]
    hyper = ~(ke + me <= 64.0 * x[:, 4])
    assert 0.05 < hyper.mean() < 0.95, hyper.mean()
    assert _bits_equal(g[hyper], x[hyper])
    cheap = ~hyper
    assert np.array_equal(g[cheap][:, [0, 5, 6, 7]], x[cheap][:, [0, 5, 6, 7]])
    gu, xu = g[cheap][:, 1:4], x[cheap][:, 1:4]
    assert (np.abs(gu.view(np.int64) - xu.view(np.int64))[xu != 0] <= 4).all()
    assert np.max(np.abs(g[cheap][:, 4] - x[cheap][:, 4]) / x[cheap][:, 4]) <= 1e-13
