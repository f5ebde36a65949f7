"""Python front of the solve server (setb_server_*, include/setb200.h): submit requests, wait for
results, drive a Poisson request stream, and the one-at-a-time baseline.

The server loop itself is native (set_b200/csrc/serve.cu): a C++ thread owns a batch and admits,
steps, checks and retires solves; this module only submits and collects.
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import Batch, Request, Result, SetbError, StepOpts, _check, _p, lib


class Server:
    def __init__(self, max_slots: int = 256, precision: int = 1, hbm_budget: int = 150 * 10 ** 9,
                 check_every: int = 50):
        h = C.c_void_p()
        _check(lib().setb_server_create(C.byref(h), int(max_slots), int(precision), int(hbm_budget),
                                        int(check_every)), "setb_server_create")
        self.h = h
        self.check_every = check_every
        self._keep = {}   # result buffers that must outlive their request

    def submit(self, inst, steady_tol: float = 1e-5, max_steps: int | None = None, keep_state: bool = False) -> int:
        r = Request()
        r.desc, r.ic, r.opts = inst.desc, inst.ic, inst.opts
        r.max_steps = int(max_steps if max_steps is not None else inst.steps)
        r.reserved = 0
        r.steady_tol = float(steady_tol)
        buf = None
        if keep_state:
            buf = np.zeros((8, inst.desc.nz, inst.desc.ny, inst.desc.nx))
            r.result_U = _p(buf)
        rid = C.c_int64()
        _check(lib().setb_server_submit(self.h, C.byref(r), C.byref(rid)), "setb_server_submit")
        if buf is not None:
            self._keep[rid.value] = buf
        return rid.value

    def wait(self, rid: int, timeout: float = 3600.0):
        out = Result()
        _check(lib().setb_server_wait(self.h, int(rid), C.byref(out), float(timeout)), "setb_server_wait")
        return out, self._keep.pop(rid, None)

    def stats(self):
        p, a, mx = C.c_int32(), C.c_int32(), C.c_int32()
        c, f = C.c_int64(), C.c_int64()
        _check(lib().setb_server_stats(self.h, C.byref(p), C.byref(a), C.byref(c), C.byref(f), C.byref(mx)),
               "setb_server_stats")
        return {"pending": p.value, "active": a.value, "completed": c.value, "failed": f.value,
                "max_active": mx.value}

    def close(self):
        if self.h:
            lib().setb_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def warm_kernels(requests, precision: int, check_every: int = 50):
    """One untimed short solve (one check interval) per distinct solver option set of the stream,
    so a timed run does not pay the kernels' first-use loading."""
    seen = set()
    for rq in requests:
        o = rq.inst.opts
        key = (o.n_state, o.n_disc, o.order, o.scheme)
        if key not in seen:
            seen.add(key)
            solve_alone(rq.inst, precision, rq.steady_tol, check_every, check_every)


def run_stream(requests, max_slots: int = 256, precision: int = 1, hbm_budget: int = 150 * 10 ** 9,
               check_every: int = 50, keep=(), warm: bool = True):
    """Submits each request at its arrival time (seconds from the start) and waits for all.
    Returns latencies (done - submit, server clock), solves/s over the stream, and results.
    `warm`: the kernels are loaded by untimed short solves first (as for run_sequential)."""
    keep = set(keep)
    if warm:
        warm_kernels(requests, precision, check_every)
    with Server(max_slots, precision, hbm_budget, check_every) as srv:
        t0 = time.perf_counter()
        ids = []
        for k, rq in enumerate(requests):
            delay = rq.arrival - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            ids.append(srv.submit(rq.inst, rq.steady_tol, rq.max_steps, keep_state=k in keep))
        results, states = [], {}
        for k, rid in enumerate(ids):
            res, U = srv.wait(rid)
            results.append(res)
            if U is not None:
                states[k] = U
        stats = srv.stats()
    lat = np.array([r.t_done - r.t_submit for r in results])
    span = max(r.t_done for r in results) - min(r.t_submit for r in results)
    failed_by_status = {}
    for r in results:
        if r.status != 0:
            name = lib().setb_strerror(int(r.status)).decode()
            failed_by_status[name] = failed_by_status.get(name, 0) + 1
    return {"latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
            "solves_per_s": len(results) / span, "span_s": span, "results": results, "states": states,
            "max_active": stats["max_active"], "failed": stats["failed"], "failed_by_status": failed_by_status,
            "steps": [r.steps for r in results], "converged": int(sum(r.converged for r in results))}


def solve_alone(inst, precision: int = 0, steady_tol: float = 1e-5, max_steps: int | None = None,
                check_every: int = 50, keep_state: bool = False):
    """One request by itself (a one-slot batch, same checks and stopping rule as the server: it
    stops at the first check that finds it steady, past its cap, or failed; `status` is the
    setb status the server would report)."""
    o = StepOpts()
    o.n_state, o.n_disc, o.order, o.scheme, o.precision, o.reserved, o.cfl = (
        inst.opts.n_state, inst.opts.n_disc, inst.opts.order, inst.opts.scheme, precision, 0, inst.opts.cfl)
    cap = max_steps if max_steps is not None else inst.steps
    status = 0
    with Batch(1, precision=precision) as b:
        s = b.add(inst.desc, inst.ic, o)
        b.check()
        steps, conv, last = 0, False, -1.0
        while steps < cap:
            b.step(check_every)
            steps += check_every
            last = b.check()[s]
            try:
                b.status(s)
            except SetbError as e:
                status = e.code
                break
            if steady_tol > 0 and 0 <= last < steady_tol:
                conv = True
                break
        U = b.conserved(s) if keep_state else None
        d = b.status(s, check=False)
    return {"steps": steps, "converged": conv, "last_change": last, "U": U, "diag": d, "status": status}


def run_sequential(requests, precision: int = 0, check_every: int = 50, warm: bool = True):
    """The same requests processed one at a time, back to back (arrival gaps ignored).  `warm`:
    untimed short solves first (warm_kernels)."""
    if warm:
        warm_kernels(requests, precision, check_every)
    t0 = time.perf_counter()
    out = [solve_alone(rq.inst, precision, rq.steady_tol, rq.max_steps, check_every) for rq in requests]
    secs = time.perf_counter() - t0
    return {"solves_per_s": len(requests) / secs, "seconds": secs, "steps": [o["steps"] for o in out]}
