"""chlld_Q (SET_Fortran_Cuda_MHD/Solvers.f90:198-1141), the passive-scalar flux routine, on the CPU.

Oracle: its HLL branch is pinned against the reference's own compiled HLL solver (the golden
vectors of SET_Gelios/source/Solvers.cpp:92-691), and it reproduces chlld bit for bit where the
two routines share their arithmetic; the scalar parts are checked by the properties the
algorithm has (a scalar equal to rho is advected exactly like rho, the konvect_ scalar and Q take
the same path, mirror symmetry).  Product: the host entry point setb_chlld_q matches the oracle
to |dF| <= 1e-12 max|F| (reciprocals instead of divisions, no tangent rotation inside the solver).
"""
import os

import numpy as np
import pytest

import oracle as O
import set_b200 as S

GOLD = os.path.join(os.path.dirname(__file__), "golden", "gelios_hll.npz")


def rand_state9(rng, bscale=2.0):
    return np.array([rng.uniform(0.1, 4.0), *rng.normal(0, 1.5, 3), rng.uniform(0.05, 4.0),
                     *rng.normal(0, bscale, 3), rng.uniform(-1.0, 2.0)])


def rand_normal(rng):
    n = rng.normal(size=3)
    return n / np.linalg.norm(n)


# ------------------------------------------------------------------ oracle pins
def test_oracle_hll_branch_matches_reference_golden_vectors():
    """The HLL branch of chlld_Q shares chlld's set-up and HLL arithmetic (n_disc 0, no ydar):
    the reference's compiled HLL solver pins its 8 MHD fluxes bit for bit."""
    g = np.load(GOLD)
    for k in range(g["q1"].shape[0]):
        q1 = np.r_[g["q1"][k], 0.5]
        q2 = np.r_[g["q2"][k], 1.5]
        rc, f, sl, sp, sc, _ = O.chlld_q(1, g["normal"][k], g["w"][k], q1, q2)
        assert rc == 0
        np.testing.assert_array_equal(f[:8], g["qqq"][k])
        assert (sl, sp, sc) == tuple(g["speeds"][k])


@pytest.mark.parametrize("n_state", [0, 1])
@pytest.mark.parametrize("n_disc", [0, 1])
def test_oracle_hll_equals_chlld_bitwise(n_state, n_disc):
    rng = np.random.default_rng(40 + n_state + 2 * n_disc)
    for t in range(300):
        q1, q2 = rand_state9(rng), rand_state9(rng)
        n = rand_normal(rng)
        w = float(rng.normal()) if t % 2 else 0.0
        rc, f, sl, sp, sc, _ = O.chlld_q(n_state, n, w, q1, q2, n_disc=n_disc)
        rc8, f8, sl8, sp8, sc8 = O.chlld(n_state, n, w, q1[:8], q2[:8], n_disc=n_disc)
        assert rc == 0 and rc8 == 0
        np.testing.assert_array_equal(f[:8], f8)
        assert (sl, sp, sc) == (sl8, sp8, sc8)


@pytest.mark.parametrize("n_state", [2, 3])
def test_oracle_star_branches_agree_with_chlld_to_rounding(n_state):
    """HLLC / HLLD of chlld_Q differ from chlld only where its constants differ (epsb 1e-4, the
    HLLC star pressure formula): away from |Bn| ~ 1e-4 the fluxes agree to rounding."""
    rng = np.random.default_rng(50 + n_state)
    for t in range(300):
        b = 0.0 if (n_state == 2 and t % 2) else 2.0
        q1, q2 = rand_state9(rng, b), rand_state9(rng, b)
        n = rand_normal(rng)
        rc, f, *_ = O.chlld_q(n_state, n, 0.0, q1, q2)
        rc8, f8, *_ = O.chlld(n_state, n, 0.0, q1[:8], q2[:8])
        assert rc == 0 and rc8 == 0
        assert np.abs(f[:8] - f8).max() <= 1e-9 * np.abs(f8).max()


@pytest.mark.parametrize("n_state", [0, 1, 2, 3])
def test_oracle_scalar_equal_to_density_is_advected_as_density(n_state):
    rng = np.random.default_rng(60 + n_state)
    for t in range(200):
        q1, q2 = rand_state9(rng), rand_state9(rng)
        q1[8], q2[8] = q1[0], q2[0]
        n = rand_normal(rng)
        w = float(rng.normal()) if t % 3 == 0 else 0.0
        rc, f, *_ = O.chlld_q(n_state, n, w, q1, q2, n_disc=t % 3, ydar=bool(t % 5 == 0))
        assert rc == 0
        assert f[8] == f[0]


@pytest.mark.parametrize("n_state", [0, 1, 2, 3])
def test_oracle_konvect_scalar_takes_the_q_path(n_state):
    rng = np.random.default_rng(70 + n_state)
    for t in range(200):
        q1, q2 = rand_state9(rng), rand_state9(rng)
        n = rand_normal(rng)
        w = float(rng.normal()) if t % 3 == 0 else 0.0
        rc, f, _, _, _, kf = O.chlld_q(n_state, n, w, q1, q2, n_disc=t % 3, ydar=bool(t % 4 == 0),
                                        konvect=(q1[8], q2[8]))
        assert rc == 0
        if w == 0.0:
            assert kf == f[8]
        else:   # the face-speed term is written wv*k*suLm for konvect_, wv*(q*suLm) for Q
            assert abs(kf - f[8]) <= 1e-14 * max(1.0, np.abs(f).max())
        # konvect_ is an extra output only: the 9 fluxes do not depend on it
        rc, g, *_ = O.chlld_q(n_state, n, w, q1, q2, n_disc=t % 3, ydar=bool(t % 4 == 0))
        np.testing.assert_array_equal(f, g)


@pytest.mark.parametrize("n_state", [1, 2, 3])
def test_oracle_mirror_symmetry(n_state):
    rng = np.random.default_rng(80 + n_state)
    for t in range(200):
        q1, q2 = rand_state9(rng), rand_state9(rng)
        n = rand_normal(rng)
        rc1, f1, *_ = O.chlld_q(n_state, n, 0.0, q1, q2)
        rc2, f2, *_ = O.chlld_q(n_state, -n, 0.0, q2, q1)
        assert rc1 == 0 and rc2 == 0
        assert np.abs(f1 + f2).max() <= 1e-11 * np.abs(f1).max()


@pytest.mark.parametrize("n_state", [1, 2, 3])
def test_oracle_ydar_is_the_left_state_flux_for_a_fixed_face(n_state):
    """ydar = .True. on a fixed face (w = 0) selects FL whenever no later selection overrides it:
    for HLL and HLLC always; for HLLD the (L** | R**) and (R* | R) selections still override it,
    so the result is either FL or the flux without ydar."""
    rng = np.random.default_rng(90 + n_state)
    n_left = 0
    for t in range(300):
        q1, q2 = rand_state9(rng), rand_state9(rng)
        n = rand_normal(rng)
        rc, f, *_ = O.chlld_q(n_state, n, 0.0, q1, q2, ydar=True)
        assert rc == 0
        _, fL, *_ = O.chlld_q(n_state, n, 0.0, q1, q1)   # consistency: F(UL, UL) = FL
        _, f0, *_ = O.chlld_q(n_state, n, 0.0, q1, q2)
        hyd = [0, 1, 2, 3, 4, 8]   # the Bn flux is not FL's (it is -max|S| dBn)
        is_left = np.abs(f[hyd] - fL[hyd]).max() <= 1e-12 * np.abs(fL).max()
        if n_state == 3 and not is_left:
            np.testing.assert_array_equal(f, f0)
        else:
            assert is_left
            n_left += 1
    assert n_left > 100


# ------------------------------------------------------------------ product, host entry point
@pytest.mark.parametrize("n_state", [0, 1, 2, 3])
@pytest.mark.parametrize("ydar", [False, True])
def test_host_chlld_q_matches_oracle(n_state, ydar):
    rng = np.random.default_rng(200 + n_state + 10 * ydar)
    for t in range(200):
        b = 0.0 if (n_state == 2 and t % 2) else 2.0
        q1, q2 = rand_state9(rng, b), rand_state9(rng, b)
        n = rand_normal(rng)
        w = float(rng.normal()) if t % 3 == 0 else 0.0
        nd = t % 3
        kv = (float(rng.normal()), float(rng.normal()))
        f, sl, sp, sc, kf = S.chlld_q(n_state, n, w, q1, q2, n_disc=nd, ydar=ydar, konvect=kv)
        rc, g, osl, osp, osc, okf = O.chlld_q(n_state, n, w, q1, q2, n_disc=nd, ydar=ydar, konvect=kv)
        assert rc == 0
        scale = max(np.abs(g).max(), abs(okf))
        assert np.abs(f - g).max() <= 1e-12 * scale, (t, f, g)
        assert abs(kf - okf) <= 1e-12 * scale
        for a, b_ in ((sl, osl), (sp, osp), (sc, osc)):
            assert abs(a - b_) <= 1e-12 * max(abs(b_), 1.0)


def test_host_chlld_q_reference_golden_hll():
    g = np.load(GOLD)
    for k in range(g["q1"].shape[0]):
        f, *_ = S.chlld_q(1, g["normal"][k], g["w"][k], np.r_[g["q1"][k], 1.0], np.r_[g["q2"][k], 2.0])
        ref = g["qqq"][k]
        assert np.abs(f[:8] - ref).max() <= 1e-12 * np.abs(ref).max()


def test_host_chlld_q_inert_and_optional_arguments():
    """null_bn1 and p_correct_ change nothing (Solvers.f90:266-267); absent OPTIONALs are the
    defaults n_disc = 0, ydar = .False.; a missing konvect_ leaves the 9 fluxes unchanged."""
    rng = np.random.default_rng(9)
    for t in range(50):
        q1, q2 = rand_state9(rng), rand_state9(rng)
        n = rand_normal(rng)
        ref, *_ = S.chlld_q(3, n, 0.0, q1, q2)
        for kw in ({"null_bn": True}, {"p_correct": True}, {"n_disc": 0, "ydar": False},
                   {"konvect": (0.3, -0.2)}, {"null_bn": False, "p_correct": False}):
            f, *_ = S.chlld_q(3, n, 0.0, q1, q2, **kw)
            np.testing.assert_array_equal(f, ref)


def test_host_chlld_q_rejects_bad_arguments():
    q = np.array([1.0, 0, 0, 0, 1.0, 0, 0, 0, 1.0])
    for ns, nd in ((4, 0), (-1, 0), (3, 3)):
        with pytest.raises(S.SetbError) as e:
            S.chlld_q(ns, (1.0, 0.0, 0.0), 0.0, q, q, n_disc=nd)
        assert e.value.code == 1
    with pytest.raises(ValueError):
        S.chlld_q(3, (1.0, 0.0, 0.0), 0.0, q[:8], q[:8])


def test_batch_entry_point_checks_arguments_on_the_host():
    """setb_chlld_q_batch validates its options before touching a device; an empty batch is a
    no-op; without a GPU a valid batch reports ENODEV (8), never a CPU result."""
    import ctypes as C
    from tests.conftest import has_gpu
    L = S.lib()
    q = np.zeros((1, 9))
    nr = np.array([[1.0, 0.0, 0.0]])
    out, sp, fl = np.zeros((1, 9)), np.zeros((1, 3)), np.zeros(1, dtype=np.int32)
    P = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    args = lambda n, ns, nd: (n, ns, nd, 0, P(nr), None, P(q), P(q), None, P(out), P(sp),
                              fl.ctypes.data_as(C.POINTER(C.c_int32)))
    assert L.setb_chlld_q_batch(*args(0, 3, 0)) == 0
    for bad in ((1, 4, 0), (1, 3, 3), (-1, 3, 0)):
        assert L.setb_chlld_q_batch(*args(*bad)) == 1
    if not has_gpu():
        assert L.setb_chlld_q_batch(*args(1, 3, 0)) == 8
