"""The z-slab decomposition of one Cartesian grid (setb_init_slab / setb_slab_stage), checked on one
GPU: all slabs of the grid run in one process with device copies for the ghost-plane exchange
(LocalSlabs), and must reproduce the single-grid solve (setb_step) bit for bit -- state, simulated
time and the whole-grid index of a bad cell -- for the plain and mixed forms, Euler and Heun,
HLLD and HLLC, even and uneven slabs, and slabs that contain the source sphere."""
import numpy as np
import pytest

import set_b200 as S
from set_b200 import slab as SL

pytestmark = pytest.mark.gpu


def whole_and_slabs(desc, cp, opts, parts, nsteps):
    with S.Solver(desc, cell_par=cp) as g:
        g.step(nsteps, opts)
        Ug, (_, tg), dg = g.conserved(), g.get_state(), g.status()
    with SL.LocalSlabs(desc, parts, cp) as ls:
        ls.step(nsteps, opts)
        Us, (_, ts) = ls.conserved(), ls.get_state()
        ds = [s.status() for s in ls.slabs]
    return Ug, tg, dg, Us, ts, ds


@pytest.mark.parametrize("shape,parts,opts", [
    ((40, 36, 30), 3, dict(n_state=3, order=2, scheme=2)),
    ((40, 36, 30), 4, dict(n_state=3, order=2, scheme=2, precision=1)),
    ((33, 29, 23), 5, dict(n_state=2, order=2, scheme=2)),
    ((32, 24, 20), 2, dict(n_state=3, order=1, scheme=1)),
])
def test_slabs_reproduce_the_single_grid_bitwise(shape, parts, opts):
    desc = S.cart_desc(shape, r_src=0.3, rho_src=20.0, dt_init=1e-3)
    lism = S.lism_prim() if opts["n_state"] == 3 else S.lism_prim(bmag=0.0)
    cp = S.fill_lism(desc, S.lism_ic(lism=lism, seed=7, pert_amp=0.05))
    o = S.step_opts(cfl=0.4, **opts)
    Ug, tg, dg, Us, ts, ds = whole_and_slabs(desc, cp, o, parts, 12)
    assert np.isfinite(Ug).all()
    assert np.array_equal(Ug, Us)
    assert tg == ts
    assert dg.n_negdens == sum(d.n_negdens for d in ds) == 0
    # every slab reports the same clock
    assert len({(d.time_all, d.dt_next, d.steps) for d in ds}) == 1


def test_slab_state_round_trip_and_step_refused():
    desc = S.cart_desc((24, 20, 16), dt_init=1e-3)
    cp = S.fill_lism(desc, S.lism_ic(seed=3))
    plane = 24 * 20
    with S.Solver(desc, cell_par=cp) as g:
        whole, _ = g.get_state()
        Uw = g.conserved()
    with SL.SlabSolver(desc, 5, 6, cp[5 * plane:11 * plane]) as s:
        out, t = s.get_state()   # the same conversions as the whole-grid handle, owned planes only
        assert np.array_equal(out[:, :8], whole[5 * plane:11 * plane, :8]) and t == 0.0
        assert np.array_equal(s.conserved(), Uw[:, 5:11])
        with pytest.raises(RuntimeError):
            s.step(1, S.step_opts())
        assert S.lib().setb_step(s.h, 1, S.step_opts(), None) == 1
        with pytest.raises(S.SetbError):
            s.stage(2, S.step_opts(scheme=1))
