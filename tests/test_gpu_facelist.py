"""Face-list path on the GPU through the C ABI (setb_init_facelist + setb_step) against the
oracle's face-list driver: per-step parity, multi-step L1, numbering invariance, determinism."""
import numpy as np
import pytest

import oracle as O
from set_b200 import facelist as FL
import set_b200 as S

pytestmark = pytest.mark.gpu


def oracle_run(m, params, cp, opts, nsteps):
    om = O.facelist(m, params)
    U = O.cellpar_to_cons(cp, (m.n_cell,)).reshape(8, -1).copy()
    ck, dg, _ = O.fl_run(om, opts, U, nsteps)
    return U, ck, dg


def gpu_run(m, params, cp, opts, nsteps):
    with FL.FaceListSolver(m, cp, params) as s:
        t = s.step(nsteps, opts)
        return s.conserved(), t, s.status()


CASES = [
    # shape, stretch, permute, n_state, order, scheme, sides, skip / freeze radii
    ((12, 10, 9), 0.5, 5, 3, 2, 2, None, (0.0, 0.0)),
    ((11, 9, 10), 0.3, None, 2, 2, 2, None, (0.0, 0.0)),
    ((10, 10, 10), 0.6, 8, 3, 1, 1, {"x+": 2, "z-": 5}, (0.0, 0.0)),
    ((12, 12, 12), 0.2, 3, 3, 2, 2, None, (0.15, 0.2)),
]


@pytest.mark.parametrize("shape,stretch,perm,n_state,order,scheme,sides,radii", CASES)
def test_facelist_matches_oracle(shape, stretch, perm, n_state, order, scheme, sides, radii):
    m = FL.box_facelist(shape, stretch=stretch, permute_seed=perm, sides=sides, seed=1)
    params = FL.fl_params(r_src=0.3, rho_src=20.0, v_src=3.0, dt_init=1e-3, face_skip_radius=radii[0],
                          cell_freeze_radius=radii[1])
    lism = S.lism_prim() if n_state == 3 else S.lism_prim(bmag=0.0)
    cp = FL.lism_cellpar(m, lism=lism, seed=3, params=params)
    opts_o = O.make_opts(n_state, order, scheme, 0.4)
    opts_g = S.step_opts(n_state=n_state, order=order, scheme=scheme, cfl=0.4)
    # one step: per-cell relative agreement
    Uo, cko, _ = oracle_run(m, params, cp, opts_o, 1)
    Ug, tg, dg = gpu_run(m, params, cp, opts_g, 1)
    assert np.isfinite(Ug).all()
    rel = np.abs(Ug - Uo) / (np.abs(Uo).max(axis=1, keepdims=True) + 1e-300)
    assert rel.max() <= 1e-12, rel.max()
    assert abs(tg - cko.time_all) <= 1e-15
    # 20 steps: relative L1 of every conserved variable
    Uo, cko, dgo = oracle_run(m, params, cp, opts_o, 20)
    Ug, tg, dg = gpu_run(m, params, cp, opts_g, 20)
    l1 = np.abs(Ug - Uo).sum(1) / (np.abs(Uo).sum(1) + 1e-300)
    assert l1.max() <= 1e-10, l1
    assert abs(tg - cko.time_all) <= 1e-12 * cko.time_all
    assert dg.n_negdens == dgo.n_negdens == 0


def test_facelist_numbering_and_determinism():
    params = FL.fl_params(r_src=0.4, rho_src=10.0, dt_init=1e-3)
    a = FL.box_facelist((14, 12, 10), stretch=0.4, seed=2)
    b = FL.box_facelist((14, 12, 10), stretch=0.4, seed=2, permute_seed=17)
    cpa = FL.lism_cellpar(a, seed=4, params=params)
    key = lambda x: np.lexsort((x[:, 0], x[:, 1], x[:, 2]))
    ia, ib = key(a.cell_center), key(b.cell_center)
    cpb = np.zeros_like(cpa)
    cpb[ib] = cpa[ia]
    o = S.step_opts(n_state=3, order=2, scheme=2, cfl=0.4)
    Ua, ta, _ = gpu_run(a, params, cpa, o, 10)
    Ua2, ta2, _ = gpu_run(a, params, cpa, o, 10)
    Ub, tb, _ = gpu_run(b, params, cpb, o, 10)
    assert np.array_equal(Ua, Ua2) and ta == ta2
    assert np.array_equal(Ua[:, ia], Ub[:, ib]) and ta == tb


def test_facelist_state_round_trip_and_mixed_rejected():
    m = FL.box_facelist((8, 7, 6), stretch=0.3, seed=5)
    params = FL.fl_params(dt_init=1e-3)
    cp = FL.lism_cellpar(m, seed=6, params=params)
    with FL.FaceListSolver(m, cp, params) as s:
        back, t = s.get_state()
        assert np.allclose(back[:, :8], cp[:, :8], rtol=1e-14, atol=1e-14) and t == 0.0
        with pytest.raises(S.SetbError):
            s.step(1, S.step_opts(precision=1))


def test_grid_file_drives_the_solver(tmp_path):
    """A grid file in the reference's format, read back, gives the same solve as the arrays."""
    m = FL.box_facelist((9, 8, 7), stretch=0.3, permute_seed=2, seed=3)
    params = FL.fl_params(r_src=0.3, rho_src=10.0, dt_init=1e-3)
    cp = FL.lism_cellpar(m, seed=1, params=params)
    p = tmp_path / "FCMHD_3.bin"
    FL.write_fcmhd(p, 0.0, cp, m)
    t0, cp2, m2, _ = FL.read_fcmhd(p)
    o = S.step_opts(n_state=3, order=2, scheme=2, cfl=0.4)
    Ua, ta, _ = gpu_run(m, params, cp, o, 8)
    Ub, tb, _ = gpu_run(m2, params, cp2, o, 8)
    assert t0 == 0.0 and np.array_equal(Ua, Ub) and ta == tb


def axisym_case(seed=0, n=(24, 16, 1)):
    """A thin box about the x axis (y >= 0 is the radius; the y = 0 side is the axis, type 5),
    z faces are walls; plasma without field, two H-atom fluids in Cell_par columns 9..16."""
    sides = {"x-": 4, "x+": 4, "y-": 5, "y+": 4, "z-": 2, "z+": 2}
    m = FL.box_facelist(n, lo=(-1.0, 0.0, -0.02), hi=(1.0, 1.0, 0.02), stretch=0.3, sides=sides,
                        permute_seed=seed + 1, seed=seed)
    params = FL.fl_params(r_src=0.0, dt_init=1e-4, face_skip_radius=0.02, cell_freeze_radius=0.05, physics=1)
    rng = np.random.default_rng(seed)
    cp = FL.lism_cellpar(m, lism=S.lism_prim(bmag=0.0), seed=seed + 2, pert_amp=0.05)
    N = m.n_cell
    cp[:, 8] = rng.uniform(0.05, 0.2, N)       # rho_H3
    cp[:, 9] = rng.uniform(-2.6, -2.2, N)      # u_H3
    cp[:, 10] = rng.uniform(-0.1, 0.1, N)      # v_H3
    cp[:, 11] = rng.uniform(0.5, 1.5, N)       # T_H3
    cp[:, 12] = rng.uniform(0.01, 0.1, N)      # rho_H4
    cp[:, 13] = rng.uniform(-2.0, -1.0, N)
    cp[:, 14] = rng.uniform(-0.3, 0.3, N)
    cp[:, 15] = rng.uniform(1.0, 3.0, N)
    cp[:5, 12] = 0.0                            # below the reference's density floor
    return m, params, cp


@pytest.mark.parametrize("scheme", [2, 1])
def test_axisymmetric_charge_exchange_matches_oracle(scheme):
    m, params, cp = axisym_case(scheme)
    opts_o = O.make_opts(2, 2, scheme, 0.4)
    opts_g = S.step_opts(n_state=2, order=2, scheme=scheme, cfl=0.4)
    om = O.facelist(m, params, cell_par=cp)
    for steps, tol in ((1, 1e-12), (20, 1e-10)):
        Uo = O.cellpar_to_cons(cp, (m.n_cell,)).reshape(8, -1).copy()
        cko, dgo, _ = O.fl_run(om, opts_o, Uo, steps)
        Ug, tg, dg = gpu_run(m, params, cp, opts_g, steps)
        assert np.isfinite(Ug).all()
        l1 = np.abs(Ug - Uo).sum(1) / (np.abs(Uo).sum(1) + 1e-300)
        assert l1.max() <= tol, (steps, l1)
        assert abs(tg - cko.time_all) <= 1e-12 * cko.time_all
        assert dg.n_negdens == dgo.n_negdens == 0
    # the axisymmetric update keeps w and B at zero; charge exchange moves momentum
    assert np.abs(Ug[3]).max() == 0.0 and np.abs(Ug[5:]).max() == 0.0


@pytest.mark.parametrize("powell,order,scheme", [(1, 2, 2), (2, 2, 2), (2, 1, 1)])
def test_facelist_divb_terms_match_oracle(powell, order, scheme):
    """The div-B option (face flux Gran_POTOK(9) and the sks sources, commented out in the
    reference at cuf_solvers.cuf:433, 529-533, 729-733) on a field with nonzero divergence."""
    m = FL.box_facelist((12, 10, 9), stretch=0.5, seed=1, permute_seed=5)
    params = FL.fl_params(r_src=0.3, rho_src=20.0, v_src=3.0, dt_init=1e-3, powell=powell)
    cp = FL.lism_cellpar(m, seed=3, pert_amp=0.05, params=params)
    rng = np.random.default_rng(9)
    cp[:, 5:8] += rng.normal(0.0, 0.1, (m.n_cell, 3))
    opts_o = O.make_opts(3, order, scheme, 0.4)
    opts_g = S.step_opts(n_state=3, order=order, scheme=scheme, cfl=0.4)
    Uo, cko, _ = oracle_run(m, params, cp, opts_o, 1)
    Ug, tg, _ = gpu_run(m, params, cp, opts_g, 1)
    rel = np.abs(Ug - Uo) / (np.abs(Uo).max(axis=1, keepdims=True) + 1e-300)
    assert rel.max() <= 1e-12, rel.max()
    # the terms act: the plain run differs by far more than the tolerance
    Up, _, _ = gpu_run(m, FL.fl_params(r_src=0.3, rho_src=20.0, v_src=3.0, dt_init=1e-3), cp, opts_g, 1)
    assert (np.abs(Up - Uo) / (np.abs(Uo).max(axis=1, keepdims=True) + 1e-300)).max() > 1e-8
    Uo, cko, dgo = oracle_run(m, params, cp, opts_o, 20)
    Ug, tg, dg = gpu_run(m, params, cp, opts_g, 20)
    l1 = np.abs(Ug - Uo).sum(1) / (np.abs(Uo).sum(1) + 1e-300)
    assert l1.max() <= 1e-10, l1
    assert abs(tg - cko.time_all) <= 1e-12 * cko.time_all
    assert dg.n_negdens == dgo.n_negdens == 0
