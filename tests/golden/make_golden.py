"""Regenerates the golden flux vectors under tests/golden/ from the reference's own C++ solvers.

The reference (SergeyMSU/SET) ships no tests or golden vectors.  Three of its C++ Riemann
solvers in SET_Gelios/source/Solvers.cpp compile here; oracle/Makefile builds them from the
reference sources into oracle/_ref/libgelios_hll.so (through oracle/ref_shim.cpp).  This script
draws seeded face states and records those solvers' outputs, so the fixtures pin the oracle (and
the product) without the reference tree:

  gelios_hll.npz     HLLD_Solver_Alexashov (:92-691, HLL): chlld's shared set-up and n_state 1.
  gelios_hllc.npz    HLLC_Aleksashov (:1324-1639): chlld's n_state 2 branch with B = 0.
  korolkov_hlld.npz  HLLDQ_Korolkov (:1642-2185, metod 3): a second author's HLLD, used as a
                     tolerance cross-check of chlld's n_state 3 branch.

    make -C oracle REF=<reference tree> && python tests/golden/make_golden.py [--all]

Without --all only missing files are written (the committed ones stay byte-stable).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
import oracle  # noqa: E402

SPI4 = np.sqrt(4.0 * np.pi)


def draw_states(rng, n):
    q = np.empty((n, 8))
    q[:, 0] = rng.uniform(0.05, 5.0, n)
    q[:, 1:4] = rng.normal(0.0, 2.0, (n, 3))
    q[:, 4] = rng.uniform(0.01, 5.0, n)
    q[:, 5:8] = rng.normal(0.0, 2.0, (n, 3))
    return q


def unit(rng):
    n = rng.normal(size=3)
    return n / np.linalg.norm(n)


def axis_normal(rng):
    return np.eye(3)[rng.integers(3)] * rng.choice([-1.0, 1.0])


def make_hll(path):
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
    np.savez_compressed(path, normal=a[:, 0:3], w=a[:, 3], q1=a[:, 4:12], q2=a[:, 12:20], qqq=a[:, 20:28],
                        speeds=a[:, 28:31])
    return len(rows)


def make_hllc(path):
    """B = 0 faces on a fixed face (w = 0): axis-aligned and general normals, subsonic faces of
    both SM signs, and supersonic faces both ways (a common normal velocity added to both sides
    until SL > 0 or SR < 0)."""
    rng = np.random.default_rng(20261204)
    rows = []
    kinds = []
    while len(rows) < 800:
        kind = len(rows) % 4
        q1, q2 = draw_states(rng, 1)[0], draw_states(rng, 1)[0]
        q1[5:8] = 0.0
        q2[5:8] = 0.0
        n = axis_normal(rng) if kind in (0, 2) else unit(rng)
        if kind >= 2:   # supersonic: shift both states along the normal
            c = max(np.sqrt(5.0 / 3.0 * q1[4] / q1[0]), np.sqrt(5.0 / 3.0 * q2[4] / q2[0]))
            shift = rng.choice([-1.0, 1.0]) * (abs(q1[1:4] @ n) + abs(q2[1:4] @ n) + 2.5 * c + rng.uniform(0, 2))
            q1[1:4] += shift * n
            q2[1:4] += shift * n
        rc, _, sl, sp, sc = oracle.chlld(2, n, 0.0, q1, q2)
        if rc or sc == 0.0 or not (sl < sp):
            continue
        f5 = oracle.ref_hllc(n, q1, q2)
        rows.append(np.concatenate([n, q1, q2, f5]))
        kinds.append(kind)
    a = np.array(rows)
    np.savez_compressed(path, normal=a[:, 0:3], q1=a[:, 3:11], q2=a[:, 11:19], qqq5=a[:, 19:24],
                        kind=np.array(kinds, dtype=np.int8))
    return len(rows)


def hlld_fan(n, q1, q2, sl, sr, sm):
    """chlld's n_state 3 intermediates on an axis-aligned face (Solvers.f90:1600-1656): the HLL
    normal field bn, the star-state denominators ttL/ttR and the Alfven speeds SZL/SZR."""
    ax = int(np.argmax(np.abs(n)))
    s = n[ax]
    r1, r2 = q1[0], q2[0]
    u1, u2 = q1[1 + ax] * s, q2[1 + ax] * s
    bx1, bx2 = q1[5 + ax] * s / SPI4, q2[5 + ax] * s / SPI4
    bn = (sr * bx2 - sl * bx1) / (sr - sl)
    suL, suR = sl - u1, sr - u2
    ttL = r1 * suL * (sl - sm) - bn * bn
    ttR = r2 * suR * (sr - sm) - bn * bn
    rzL, rzR = r1 * suL / (sl - sm), r2 * suR / (sr - sm)
    szl = sm - abs(bn) / np.sqrt(rzL)
    szr = sm + abs(bn) / np.sqrt(rzR)
    return bn, ttL, ttR, szl, szr


def make_korolkov(path):
    """Axis-aligned faces, w = 0, in the two families where HLLDQ_Korolkov's wave-speed estimate
    (min(u1,u2) - max(cfL,cfR), max(u1,u2) + max(cfL,cfR)) equals chlld's n_disc = 0 estimate
    (min(u1-cfL, u2-cfR), max(u1+cfL, u2+cfR)):
      A: equal fast speeds -- the same rho, p, B_n and tangential field magnitudes (tangential
         components sign-flipped), any velocities;
      B: equal normal velocities, any densities, pressures and fields.
    Faces inside the bands where the two solvers' thresholds differ (|bn| in (1e-6, 1e-3], |tt|
    in (1e-9, 1e-6)) are skipped.  24 more faces lie in chlld's "last match wins" region
    (SL > 0 > SZL or SR < 0 < SZR), marked quirk = 1: there the two solvers select different
    fan regions (chlld's sequential IF blocks let the last match win; HLLDQ_Korolkov's else-if
    chain takes the first)."""
    rng = np.random.default_rng(20261205)
    rows, fam, quirk = [], [], []

    def add(n, q1, q2, k, q):
        f, pq = oracle.ref_korolkov(3, n, q1, q2)
        rows.append(np.concatenate([n, q1, q2, f]))
        fam.append(k)
        quirk.append(q)

    while len(rows) < 800:
        k = len(rows) % 2
        n = axis_normal(rng)
        ax = int(np.argmax(np.abs(n)))
        q1, q2 = draw_states(rng, 1)[0], draw_states(rng, 1)[0]
        if k == 0:
            q2[0], q2[4], q2[5:8] = q1[0], q1[4], q1[5:8]
            t = [i for i in range(3) if i != ax]
            flip = rng.integers(1, 4)
            if flip & 1:
                q2[5 + t[0]] = -q2[5 + t[0]]
            if flip & 2:
                q2[5 + t[1]] = -q2[5 + t[1]]
        else:
            q2[1 + ax] = q1[1 + ax]
        if len(rows) % 10 == 9:   # weak fields: chlld's bn below epsb as well
            q1[5:8] *= 1e-8
            q2[5:8] *= 1e-8
        rc, _, sl, sp, sc = oracle.chlld(3, n, 0.0, q1, q2)
        if rc:
            continue
        bn, ttL, ttR, szl, szr = hlld_fan(n, q1, q2, sl, sp, sc)
        if 1e-6 < abs(bn) <= 1e-3 or any(1e-9 < abs(t) < 1e-6 for t in (ttL, ttR)):
            continue
        if (sl > 0 > szl) or (sp < 0 < szr):
            continue
        add(n, q1, q2, k, 0)
    # the "last match wins" region, both sides: family B faces shifted along the normal until
    # SL is just above 0 (or SR just below 0)
    for side in (0, 1):
        got = 0
        while got < 12:
            n = axis_normal(rng)
            ax = int(np.argmax(np.abs(n)))
            q1, q2 = draw_states(rng, 1)[0], draw_states(rng, 1)[0]
            q2[1 + ax] = q1[1 + ax]
            rc, _, sl, sp, sc = oracle.chlld(3, n, 0.0, q1, q2)
            sh = (-sl + rng.uniform(0, 0.3)) if side == 0 else (-sp - rng.uniform(0, 0.3))
            q1[1:4] += sh * n
            q2[1:4] += sh * n
            rc, _, sl, sp, sc = oracle.chlld(3, n, 0.0, q1, q2)
            if rc:
                continue
            bn, ttL, ttR, szl, szr = hlld_fan(n, q1, q2, sl, sp, sc)
            if 1e-6 < abs(bn) <= 1e-3 or any(1e-9 < abs(t) < 1e-6 for t in (ttL, ttR)):
                continue
            if (side == 0 and sl > 0 > szl) or (side == 1 and sp < 0 < szr):
                add(n, q1, q2, 1, 1)
                got += 1
    a = np.array(rows)
    np.savez_compressed(path, normal=a[:, 0:3], q1=a[:, 3:11], q2=a[:, 11:19], qqq=a[:, 19:27],
                        family=np.array(fam, dtype=np.int8), quirk=np.array(quirk, dtype=np.int8))
    return len(rows)


def main():
    assert oracle.ref_available(), "oracle/_ref/libgelios_hll.so missing: make -C oracle REF=<reference tree>"
    force = "--all" in sys.argv
    for name, fn in (("gelios_hll.npz", make_hll), ("gelios_hllc.npz", make_hllc),
                     ("korolkov_hlld.npz", make_korolkov)):
        path = os.path.join(HERE, name)
        if force or not os.path.exists(path):
            print("wrote", fn(path), "cases to", name)


if __name__ == "__main__":
    main()
