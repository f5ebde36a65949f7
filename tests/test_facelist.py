"""Face-list grids on the CPU: the generator's connectivity, the oracle's face-list driver
(properties the reference's face/cell kernels imply: numbering does not matter, walls conserve
mass -- and energy without a field --, a state at rest stays at rest) and the C ABI's host-side
mesh validation."""
import numpy as np
import pytest

import oracle as O
import set_b200 as S
from set_b200 import facelist as FL


def check_connectivity(m):
    N, G = m.n_cell, m.n_gran
    cnt = np.zeros(G, int)
    for c in range(N):
        for f in m.cell_gran[c]:
            if f == 0:
                continue
            assert 1 <= f <= G
            assert c + 1 in tuple(m.gran_neighbour[f - 1])
            cnt[f - 1] += 1
    inner = m.gran_neighbour[:, 1] > 0
    assert np.all(cnt[inner] == 2) and np.all(cnt[~inner] == 1)
    d = m.cell_center[m.gran_neighbour[inner, 1] - 1] - m.cell_center[m.gran_neighbour[inner, 0] - 1]
    assert np.all((d * m.gran_normal[inner]).sum(1) > 0)
    d = m.gran_center[~inner] - m.cell_center[m.gran_neighbour[~inner, 0] - 1]
    assert np.all((d * m.gran_normal[~inner]).sum(1) > 0)


@pytest.mark.parametrize("shape,stretch,perm", [((5, 4, 3), 0.0, None), ((6, 5, 4), 0.6, 7)])
def test_box_facelist_connectivity(shape, stretch, perm):
    m = FL.box_facelist(shape, stretch=stretch, permute_seed=perm, seed=2)
    nx, ny, nz = shape
    assert m.n_cell == nx * ny * nz
    assert m.n_gran == (nx + 1) * ny * nz + nx * (ny + 1) * nz + nx * ny * (nz + 1)
    assert abs(m.cell_volume.sum() - 8.0) < 1e-12
    check_connectivity(m)


def run_oracle(m, params, cp, opts, nsteps):
    om = O.facelist(m, params)
    U = O.cellpar_to_cons(cp, (m.n_cell,)).reshape(8, -1).copy()
    ck, dg, _ = O.fl_run(om, opts, U, nsteps)
    return U, ck, dg


def test_oracle_facelist_numbering_does_not_matter():
    params = FL.fl_params(r_src=0.5, rho_src=5.0, dt_init=1e-3)
    a = FL.box_facelist((7, 6, 5), stretch=0.4, seed=3)
    b = FL.box_facelist((7, 6, 5), stretch=0.4, seed=3, permute_seed=11)
    cpa = FL.lism_cellpar(a, seed=5, params=params)
    # the same physical cell in b: match by centre
    key = lambda x: np.lexsort((x[:, 0], x[:, 1], x[:, 2]))
    ia, ib = key(a.cell_center), key(b.cell_center)
    cpb = np.zeros_like(cpa)
    cpb[ib] = cpa[ia]
    o = O.make_opts(3, 2, 2, 0.4)
    Ua, cka, _ = run_oracle(a, params, cpa, o, 6)
    Ub, ckb, _ = run_oracle(b, params, cpb, o, 6)
    assert np.array_equal(Ua[:, ia], Ub[:, ib])
    assert cka.time_all == ckb.time_all


@pytest.mark.parametrize("n_state", [2, 3])
def test_oracle_facelist_walls_conserve(n_state):
    walls = {k: 2 for k in ("x-", "x+", "y-", "y+", "z-", "z+")}
    m = FL.box_facelist((6, 5, 4), stretch=0.5, sides=walls, seed=1, permute_seed=3)
    params = FL.fl_params(r_src=0.0, dt_init=1e-3)
    cp = FL.lism_cellpar(m, seed=2, pert_amp=0.2)
    if n_state == 2:
        cp[:, 5:8] = 0.0
    U0 = O.cellpar_to_cons(cp, (m.n_cell,)).reshape(8, -1)
    U, ck, dg = run_oracle(m, params, cp, O.make_opts(n_state, 2, 2, 0.4), 10)
    vol = m.cell_volume
    # the reference's wall mirrors the velocity only, so with a field the Poynting flux crosses it:
    # mass is conserved in both cases, energy in the hydro case
    for v in ((0, 4) if n_state == 2 else (0,)):
        tot0, tot = (U0[v] * vol).sum(), (U[v] * vol).sum()
        assert abs(tot - tot0) <= 1e-13 * abs(tot0), (v, tot0, tot)
    assert dg.n_negdens == 0 and dg.n_pfloor == 0


def test_oracle_facelist_rest_state_stays():
    walls = {k: 2 for k in ("x-", "x+", "y-", "y+", "z-", "z+")}
    m = FL.box_facelist((5, 5, 5), stretch=0.3, sides=walls, seed=4)
    params = FL.fl_params(r_src=0.0, dt_init=1e-3)
    cp = FL.lism_cellpar(m, lism=np.array([1.3, 0, 0, 0, 0.7, 0.2, -0.4, 0.1]), pert_amp=0.0)
    U0 = O.cellpar_to_cons(cp, (m.n_cell,)).reshape(8, -1)
    U, _, _ = run_oracle(m, params, cp, O.make_opts(3, 2, 2, 0.4), 5)
    assert np.allclose(U, U0, rtol=0, atol=1e-14)


def test_init_facelist_validates_on_the_host():
    m = FL.box_facelist((4, 3, 3), seed=1)
    params = FL.fl_params()
    cp = FL.lism_cellpar(m)
    try:   # a valid mesh passes the host checks: it then needs a device (ENODEV without one)
        FL.FaceListSolver(m, cp, params).close()
    except S.SetbError as e:
        assert e.code == 8, e
    bad = FL.FaceList(**{k: getattr(m, k).copy() for k in m.__dataclass_fields__})
    bad.gran_neighbour[5, 0] = m.n_cell + 7          # a cell number outside the grid
    with pytest.raises(S.SetbError) as e:
        FL.FaceListSolver(bad, cp, params)
    assert e.value.code == 1
    bad = FL.FaceList(**{k: getattr(m, k).copy() for k in m.__dataclass_fields__})
    bad.gran_type[3] = 9                               # unknown face type
    with pytest.raises(S.SetbError) as e:
        FL.FaceListSolver(bad, cp, params)
    assert e.value.code == 1
    bad = FL.FaceList(**{k: getattr(m, k).copy() for k in m.__dataclass_fields__})
    inner = np.where(bad.gran_neighbour[:, 1] > 0)[0][0]
    bad.gran_neighbour[inner, 1] = -1                  # a missing neighbour on an ordinary face
    bad.gran_type[inner] = 1
    with pytest.raises(S.SetbError) as e:
        FL.FaceListSolver(bad, cp, params)
    assert e.value.code == 1


def test_axisymmetric_physics_needs_positive_radius():
    m = FL.box_facelist((4, 3, 2), lo=(-1.0, -0.5, -0.1), hi=(1.0, 0.5, 0.1), seed=1)
    cp = FL.lism_cellpar(m)
    with pytest.raises(S.SetbError) as e:
        FL.FaceListSolver(m, cp, FL.fl_params(physics=1))
    assert e.value.code == 1
    with pytest.raises(S.SetbError) as e:
        FL.FaceListSolver(m, cp, FL.fl_params(physics=2))
    assert e.value.code == 1


def test_oracle_source_mk_moves_plasma_towards_the_atoms():
    """Charge exchange in the oracle's axisymmetric update: with fast H atoms along +x and the
    plasma at rest, the plasma's x momentum grows (Source_MK, cuf_kernel.cuf:215-288)."""
    m = FL.box_facelist((6, 5, 1), lo=(-1.0, 0.1, -0.02), hi=(1.0, 1.0, 0.02), seed=1,
                        sides={"x-": 2, "x+": 2, "y-": 2, "y+": 2, "z-": 2, "z+": 2})
    params = FL.fl_params(r_src=0.0, dt_init=1e-3, physics=1)
    cp = FL.lism_cellpar(m, lism=np.array([1.0, 0, 0, 0, 1.0, 0, 0, 0]), pert_amp=0.0)
    cp[:, 8:12] = [0.2, 3.0, 0.0, 1.0]
    cp[:, 12:16] = [0.0, 0.0, 0.0, 1.0]
    om = O.facelist(m, params, cell_par=cp)
    U = O.cellpar_to_cons(cp, (m.n_cell,)).reshape(8, -1).copy()
    O.fl_run(om, O.make_opts(2, 1, 1, 0.4), U, 1)
    assert (U[1] > 0).all()


def _nonsolenoidal_cellpar(m, seed):
    cp = FL.lism_cellpar(m, seed=seed, pert_amp=0.05)
    rng = np.random.default_rng(seed + 100)
    cp[:, 5:8] += rng.normal(0.0, 0.3, (m.n_cell, 3))   # random B: div B != 0 in every cell
    return cp


def _sks(m, divb):
    """Owner-signed sum of the div-B face fluxes over each cell's faces (cuf_solvers.cuf:691-703)."""
    s = np.zeros(m.n_cell)
    for c in range(m.n_cell):
        for j in m.cell_gran[c]:
            if j == 0:
                continue
            s[c] += divb[j - 1] if m.gran_neighbour[j - 1, 0] == c + 1 else -divb[j - 1]
    return s


def test_oracle_divb_face_flux_is_the_commented_expression():
    """Gran_POTOK(9) with the div-B terms on: 0.5 * n.(B1 + B2) * square of the states given to
    chlld (cuf_solvers.cuf:433, commented there); a ghost face's second state carries B1."""
    m = FL.box_facelist((5, 4, 4), stretch=0.4, seed=2, permute_seed=6)
    cp = _nonsolenoidal_cellpar(m, 3)
    om = O.facelist(m, FL.fl_params(r_src=0.0, dt_init=1e-4, powell=1))
    U = O.cellpar_to_cons(cp, (m.n_cell,)).reshape(8, -1).copy()
    _, _, flux = O.fl_run(om, O.make_opts(3, 1, 1, 0.4), U, 1)
    B = cp[:, 5:8]
    s1 = m.gran_neighbour[:, 0] - 1
    s2 = np.where(m.gran_neighbour[:, 1] > 0, m.gran_neighbour[:, 1] - 1, s1)
    n, bs = m.gran_normal, B[s1] + B[s2]
    want = 0.5 * ((n[:, 0] * bs[:, 0] + n[:, 1] * bs[:, 1]) + n[:, 2] * bs[:, 2]) * m.gran_square
    np.testing.assert_array_equal(flux[:, 8], want)
    # off (the reference's live code): zero
    _, _, flux0 = O.fl_run(O.facelist(m, FL.fl_params(r_src=0.0, dt_init=1e-4)), O.make_opts(3, 1, 1, 0.4),
                           O.cellpar_to_cons(cp, (m.n_cell,)).reshape(8, -1).copy(), 1)
    assert not flux0[:, 8].any()


@pytest.mark.parametrize("powell", [1, 2])
def test_oracle_powell_sources_match_their_definition(powell):
    """One forward-Euler step: the div-B run differs from the plain one by -dt/V times
    (0, B/4pi sks, [u.B/4pi sks], u sks); rho (and E without the energy term) bit for bit."""
    m = FL.box_facelist((6, 5, 4), stretch=0.3, seed=4)
    cp = _nonsolenoidal_cellpar(m, 5)
    o = O.make_opts(3, 1, 1, 0.4)
    U0 = O.cellpar_to_cons(cp, (m.n_cell,)).reshape(8, -1)
    Up, Uq = U0.copy(), U0.copy()
    dt = 1e-4
    O.fl_run(O.facelist(m, FL.fl_params(r_src=0.0, dt_init=dt)), o, Up, 1)
    _, _, flux = O.fl_run(O.facelist(m, FL.fl_params(r_src=0.0, dt_init=dt, powell=powell)), o, Uq, 1)
    sks = _sks(m, flux[:, 8])
    assert np.abs(sks).max() > 1e-3
    u, B = cp[:, 1:4], cp[:, 5:8]
    src = np.zeros((8, m.n_cell))
    src[1:4] = (B / (4 * np.pi) * sks[:, None]).T
    src[5:8] = (u * sks[:, None]).T
    if powell == 2:
        src[4] = (u * B).sum(1) / (4 * np.pi) * sks
    d = Uq - Up
    want = -dt * src / m.cell_volume
    scale = np.maximum(np.abs(U0).max(axis=1, keepdims=True), 1e-3)   # w = 0 in the LISM state
    assert (np.abs(d - want) / scale).max() <= 1e-13
    np.testing.assert_array_equal(Uq[0], Up[0])
    if powell == 1:
        np.testing.assert_array_equal(Uq[4], Up[4])


def test_oracle_powell_vanishes_with_a_uniform_field():
    """A uniform field has no divergence: over one forward-Euler stage (the field is uniform in
    its input) the div-B terms change nothing beyond rounding; the closed cells' outward area
    vectors sum to zero."""
    m = FL.box_facelist((6, 5, 5), stretch=0.5, seed=7)
    cp = FL.lism_cellpar(m, seed=8, pert_amp=0.05)     # uniform B, perturbed rho and p
    o = O.make_opts(3, 2, 1, 0.4)
    U0 = O.cellpar_to_cons(cp, (m.n_cell,)).reshape(8, -1)
    Up, Uq = U0.copy(), U0.copy()
    O.fl_run(O.facelist(m, FL.fl_params(r_src=0.0, dt_init=1e-3)), o, Up, 1)
    O.fl_run(O.facelist(m, FL.fl_params(r_src=0.0, dt_init=1e-3, powell=2)), o, Uq, 1)
    assert (np.abs(Uq - Up) / np.maximum(np.abs(U0).max(axis=1, keepdims=True), 1e-3)).max() <= 1e-12


def test_powell_option_is_validated_on_the_host():
    m = FL.box_facelist((4, 3, 2), lo=(-1.0, 0.1, -0.1), hi=(1.0, 1.0, 0.1), seed=1)
    cp = FL.lism_cellpar(m)
    for params in (FL.fl_params(powell=3), FL.fl_params(powell=-1), FL.fl_params(physics=1, powell=1)):
        with pytest.raises(S.SetbError) as e:
            FL.FaceListSolver(m, cp, params)
        assert e.value.code == 1


@pytest.mark.parametrize("powell", [1, 2])
def test_oracle_powell_keeps_mass_conservation(powell):
    """The div-B sources act on momentum, B (and energy) only: in a closed box mass is conserved
    to round-off over Heun steps with a non-solenoidal field."""
    walls = {k: 2 for k in ("x-", "x+", "y-", "y+", "z-", "z+")}
    m = FL.box_facelist((6, 5, 4), stretch=0.4, sides=walls, seed=3, permute_seed=2)
    cp = _nonsolenoidal_cellpar(m, 4)
    U0 = O.cellpar_to_cons(cp, (m.n_cell,)).reshape(8, -1)
    U = U0.copy()
    _, dg, _ = O.fl_run(O.facelist(m, FL.fl_params(r_src=0.0, dt_init=1e-3, powell=powell)),
                        O.make_opts(3, 2, 2, 0.4), U, 8)
    tot0, tot = (U0[0] * m.cell_volume).sum(), (U[0] * m.cell_volume).sum()
    assert abs(tot - tot0) <= 1e-13 * abs(tot0)
    assert dg.n_negdens == 0
