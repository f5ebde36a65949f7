"""The solve server (continuous batching): requests arriving while others run are admitted as
memory frees up, and each result is bit-identical to the same request solved alone (a one-solve
batch with the same checks and stopping rule)."""
import time

import numpy as np
import pytest

import set_b200 as S
from set_b200 import serve, workloads

pytestmark = pytest.mark.gpu


def small_stream(n=6, seed=11):
    reqs = workloads.c5_requests(count=n, rate=40.0, seed=seed, lo=20, hi=40, max_steps=150)
    for r in reqs:
        r.max_steps = 150
    return reqs


def test_served_results_equal_alone():
    reqs = small_stream()
    out = serve.run_stream(reqs, max_slots=8, precision=1, keep=range(len(reqs)))
    assert out["failed"] == 0 and out["max_active"] >= 2   # work overlapped on the device
    for k, rq in enumerate(reqs):
        alone = serve.solve_alone(rq.inst, precision=1, steady_tol=rq.steady_tol, max_steps=rq.max_steps,
                                  keep_state=True)
        res = out["results"][k]
        assert res.steps == alone["steps"]
        np.testing.assert_array_equal(out["states"][k], alone["U"])


def test_admission_waits_for_room():
    reqs = small_stream(5, seed=12)
    sizes = [r.inst.cells for r in reqs]
    # a budget that holds the two largest solves at most
    with S.Batch(2) as probe:
        big = sorted(range(len(reqs)), key=lambda k: -sizes[k])[:2]
        for k in big:
            probe.add(reqs[k].inst.desc, reqs[k].inst.ic, reqs[k].inst.opts)
        budget = probe.info()["bytes_used"]
    out = serve.run_stream(reqs, max_slots=8, precision=1, hbm_budget=budget)
    assert out["failed"] == 0
    assert 1 <= out["max_active"] <= 4
    assert all(r.status == 0 for r in out["results"])


def test_oversized_request_is_refused():
    reqs = small_stream(2, seed=13)
    with serve.Server(max_slots=4, precision=1, hbm_budget=1000) as srv:
        rid = srv.submit(reqs[0].inst, max_steps=50)
        res, _ = srv.wait(rid, timeout=60)
    assert res.status == 11   # SETB_EBUSY: never fits the budget


def test_steady_state_stops_early():
    reqs = small_stream(1, seed=14)
    inst = reqs[0].inst
    with serve.Server(max_slots=2, precision=1) as srv:
        rid = srv.submit(inst, steady_tol=0.5, max_steps=1000)
        res, _ = srv.wait(rid, timeout=120)
    assert res.status == 0 and res.converged == 1 and res.steps < 1000
    assert 0 <= res.last_change < 0.5
