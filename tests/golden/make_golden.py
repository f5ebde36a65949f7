"""Regenerates tests/golden/gelios_hll.npz from the reference's own C++ HLL solver.

The reference (SergeyMSU/SET) ships no tests or golden vectors.  Its C++ translation of chlld,
Solvers::HLLD_Solver_Alexashov (SET_Gelios/source/Solvers.cpp:92-691, n_state hard-wired to 1 =
HLL), compiles here; oracle/Makefile builds it from the reference sources into
oracle/_ref/libgelios_hll.so.  This script draws seeded random face states and records that
library's outputs, so the fixtures pin the oracle (and the product) without the reference tree.

    make -C oracle && python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
import oracle  # noqa: E402


def draw_states(rng, n):
    q = np.empty((n, 8))
    q[:, 0] = rng.uniform(0.05, 5.0, n)
    q[:, 1:4] = rng.normal(0.0, 2.0, (n, 3))
    q[:, 4] = rng.uniform(0.01, 5.0, n)
    q[:, 5:8] = rng.normal(0.0, 2.0, (n, 3))
    return q


def main():
    assert oracle.ref_available(), "oracle/_ref/libgelios_hll.so missing: run make -C oracle with the reference tree"
    rng = np.random.default_rng(20261203)
    rows = []
    while len(rows) < 600:
        q1, q2 = draw_states(rng, 1)[0], draw_states(rng, 1)[0]
        kind = len(rows) % 4
        if kind == 0:
            n = np.eye(3)[rng.integers(3)] * rng.choice([-1.0, 1.0])
        elif kind == 1:   # B parallel to the normal: basis fallback branch
            n = rng.normal(size=3)
            n /= np.linalg.norm(n)
            q1[5:8] = n * rng.normal()
            q2[5:8] = n * rng.normal()
        else:
            n = rng.normal(size=3)
            n /= np.linalg.norm(n)
        w = 0.0 if kind < 3 else float(rng.normal())
        # the reference function exits the process unless SL < SM < SR; screen with the oracle
        rc, _, sl, sp, sc = oracle.chlld(1, n, w, q1, q2)
        if rc or not (sl < sc < sp):
            continue
        qqq, dsl, dsp, dsc = oracle.ref_hll(n, w, q1, q2)
        rows.append(np.concatenate([n, [w], q1, q2, qqq, [dsl, dsp, dsc]]))
    a = np.array(rows)
    np.savez_compressed(os.path.join(HERE, "gelios_hll.npz"), normal=a[:, 0:3], w=a[:, 3], q1=a[:, 4:12],
                        q2=a[:, 12:20], qqq=a[:, 20:28], speeds=a[:, 28:31])
    print("wrote", len(rows), "cases")


if __name__ == "__main__":
    main()
