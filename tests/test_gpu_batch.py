"""Batched solves (setb_batch_*): per-solve results independent of the batch.

* A solve in a batch matches the same solve run alone through the single-solve handle: plain
  FP64 relative L1 <= 1e-12 per conserved variable (vector components against the vector's
  L1); mixed <= 1e-6, the mixed form's accuracy class (the same tile arithmetic compiled into a
  different kernel contracts FP32 operations differently).
* A solve alone in a batch and the same solve in a mix (with members added and removed between
  steps) are bit-identical, and so are their steady-state check values.
"""
import numpy as np
import pytest

import set_b200 as S

pytestmark = pytest.mark.gpu


def l1_vars(a, b):
    """Relative L1 per conserved variable; momentum and B components are measured against the
    whole vector's L1 (a component that is near zero everywhere has no scale of its own)."""
    d = np.abs(a - b).reshape(8, -1).sum(1)
    s = np.abs(b).reshape(8, -1).sum(1)
    s[1:4] = s[1:4].sum()
    s[5:8] = s[5:8].sum()
    return d / np.maximum(s, 1e-300)


def l1(a, b):
    return l1_vars(a, b).max()


PROBLEMS = [
    # shape, seed, n_state, inflow kwargs
    ((40, 24, 36), 1, 3, {}),
    ((33, 17, 20), 2, 3, {"tilt_deg": 20.0, "u": (-2.5, 0.0, 0.0)}),
    ((64, 32, 16), 3, 2, {"bmag": 0.0}),
    ((20, 48, 24), 4, 3, {"bmag": 1.7}),
]


def problem(k, precision):
    shape, seed, ns, kw = PROBLEMS[k]
    inflow = S.lism_prim(**kw)
    return (S.cart_desc(shape, inflow=inflow), S.lism_ic(lism=inflow, seed=seed),
            S.step_opts(n_state=ns, precision=precision))


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_matches_single_solves(precision):
    with S.Batch(8, precision=precision) as b:
        slots = [b.add(*problem(k, precision)) for k in range(len(PROBLEMS))]
        b.step(20)   # graph-replayed chunk
        b.step(5)    # directly enqueued chunk
        got = [b.conserved(s) for s in slots]
        stat = [b.status(s) for s in slots]
    tol = 1e-12 if precision == 0 else 1e-6
    for k in range(len(PROBLEMS)):
        d, ic, o = problem(k, precision)
        with S.Solver(d, ic=ic) as s:
            t = s.step(25, o)
            ref = s.conserved()
        assert l1(got[k], ref) <= tol, (k, l1_vars(got[k], ref))
        assert abs(stat[k].time_all - t) <= tol * t and stat[k].steps == 25


def test_batch_alone_and_in_mix_are_bitwise_equal():
    target = 1
    with S.Batch(4) as alone:
        s = alone.add(*problem(target, 1))
        alone.check()
        alone.step(16)
        c1 = alone.check()[s]
        alone.step(16)
        c2 = alone.check()[s]
        U_alone = alone.conserved(s)
    with S.Batch(6) as mix:
        a = mix.add(*problem(0, 1))
        s = mix.add(*problem(target, 1))
        mix.check()
        mix.step(16)
        m1 = mix.check()[s]
        mix.remove(a)                       # a member leaves ...
        c = mix.add(*problem(2, 1))         # ... and another joins between steps
        mix.step(10)
        d = mix.add(*problem(3, 1))
        mix.step(6)
        m2 = mix.check()[s]
        U_mix = mix.conserved(s)
        assert mix.status(c).steps == 16 and mix.status(d).steps == 6
    np.testing.assert_array_equal(U_mix, U_alone)
    assert (m1, m2) == (c1, c2) and c1 > 0 and c2 > 0


def test_batch_admission_by_hbm_budget():
    d, ic, o = problem(0, 1)
    with S.Batch(4, hbm_budget=1) as tiny:
        assert tiny.try_add(d, ic, o) is None
    with S.Batch(4) as probe:
        probe.add(d, ic, o)
        one = probe.info()["bytes_used"]
    with S.Batch(4, hbm_budget=one + one // 2) as b:
        s0 = b.add(d, ic, o)
        assert b.try_add(d, ic, o) is None          # the second one does not fit
        b.remove(s0)
        assert b.try_add(d, ic, o) is not None      # room again after retiring the first


def test_batch_check_is_the_density_change():
    d, ic, o = problem(0, 1)
    with S.Batch(2) as b:
        s = b.add(d, ic, o)
        assert b.check()[s] == -1.0                 # first check: no previous snapshot
        r0 = b.conserved(s)[0]
        b.step(12)
        r1 = b.conserved(s)[0]
        c = b.check()[s]
    ref = np.abs(r1 - r0).sum() / np.abs(r1).sum()
    assert abs(c - ref) <= 1e-12 * ref


def test_batch_tuning_does_not_change_results():
    out = []
    for tune in (False, True):
        with S.Batch(6) as b:
            slots = [b.add(*problem(k, 1)) for k in range(3)]
            if tune:
                t = b.tune(reps=2)
                assert t["lz"] in (8, 16, 32, 64, 1 << 20) and t["grid_mult"] in (1, 2)
            b.step(12)
            out.append([b.conserved(s) for s in slots])
            assert all(b.status(s).steps == 12 for s in slots)
    for a, c in zip(*out):
        np.testing.assert_array_equal(a, c)
