"""Host-side pieces of the product: the C ABI loads and exports every declared entry point, the
host chlld (the reference's host-callable flux routine) matches the oracle, the host initial-
condition generator matches the oracle bit for bit, and arguments are validated."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import oracle as O
import set_b200 as S
from tests.conftest import has_gpu

HEADER = os.path.join(os.path.dirname(os.path.dirname(__file__)), "include", "setb200.h")


def declared_entry_points():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"SETB_API\s+[\w\s\*]+?\b(setb_\w+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    names = declared_entry_points()
    assert len(names) >= 16
    lib = C.CDLL(S.LIB_PATH)
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) <= set(S._SIGS), set(names) - set(S._SIGS)


def rand_state(rng, bscale=2.0):
    return np.array([rng.uniform(0.1, 4.0), *rng.normal(0, 1.5, 3), rng.uniform(0.05, 4.0),
                     *rng.normal(0, bscale, 3)])


@pytest.mark.parametrize("n_state", [0, 1, 2, 3])
@pytest.mark.parametrize("moving", [False, True])
def test_host_chlld_matches_oracle(n_state, moving):
    # The product restates chlld with reciprocals and without the tangent rotation; it agrees
    # with the oracle to rounding: |dF| <= 1e-12 * max|F| per face.
    rng = np.random.default_rng(100 + n_state + 10 * moving)
    for t in range(300):
        q1, q2 = rand_state(rng, 0.0 if n_state == 2 else 2.0), rand_state(rng, 0.0 if n_state == 2 else 2.0)
        n = rng.normal(size=3)
        n /= np.linalg.norm(n)
        w = float(rng.normal()) if moving else 0.0
        f, sl, sp, sc = S.chlld(n_state, n, w, q1, q2)
        rc, g, osl, osp, osc = O.chlld(n_state, n, w, q1, q2)
        assert rc == 0
        scale = np.abs(g).max()
        assert np.abs(f - g).max() <= 1e-12 * scale, (t, f, g)
        for a, b in ((sl, osl), (sp, osp), (sc, osc)):
            assert abs(a - b) <= 1e-12 * max(abs(b), 1.0)


def test_host_chlld_reference_golden_hll():
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "gelios_hll.npz"))
    for k in range(g["q1"].shape[0]):
        f, *_ = S.chlld(1, g["normal"][k], g["w"][k], g["q1"][k], g["q2"][k])
        ref = g["qqq"][k]
        assert np.abs(f - ref).max() <= 1e-12 * np.abs(ref).max()


def test_host_chlld_reference_golden_hllc():
    """HLLC on B = 0 faces against the reference's own C++ HLLC (Solvers.cpp:1324-1639)."""
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "gelios_hllc.npz"))
    for k in range(g["q1"].shape[0]):
        f, *_ = S.chlld(2, g["normal"][k], 0.0, g["q1"][k], g["q2"][k])
        ref = g["qqq5"][k]
        assert np.abs(f[:5] - ref).max() <= 1e-12 * np.abs(ref).max()
        assert np.abs(f[5:]).max() == 0.0


def test_host_chlld_cross_check_korolkov_hlld():
    """HLLD against the reference's HLLDQ_Korolkov (metod 3) outside chlld's last-match-wins
    region: |dF| <= 1e-10 max|F| per face (the two solvers' operation orders differ)."""
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "korolkov_hlld.npz"))
    errs = []
    for k in np.nonzero(g["quirk"] == 0)[0]:
        f, *_ = S.chlld(3, g["normal"][k], 0.0, g["q1"][k], g["q2"][k])
        errs.append(np.abs(f - g["qqq"][k]).max() / np.abs(g["qqq"][k]).max())
    assert max(errs) <= 1e-10 and np.median(errs) <= 1e-14


def test_host_chlld_rejects_bad_arguments():
    q = np.array([1.0, 0, 0, 0, 1.0, 0, 0, 0])
    with pytest.raises(S.SetbError) as e:
        S.chlld(7, (1.0, 0.0, 0.0), 0.0, q, q)
    assert e.value.code == 1
    assert S.lib().setb_strerror(4) == b"cell update produced non-positive density"


@pytest.mark.parametrize("n", [(12, 10, 9), (15, 15, 15)])
def test_host_initial_condition_matches_oracle_bitwise(n):
    desc = S.cart_desc(n)
    ic = S.lism_ic(seed=9)
    cp = S.fill_lism(desc, ic)
    g = O.make_grid(n, r_floor=desc.r_floor)
    Uo = O.init_lism(g, lism=np.array(ic.lism[:]), seed=9, pert_amp=1e-3)
    Uh = O.cellpar_to_cons(cp, (desc.nz, desc.ny, desc.nx))
    np.testing.assert_array_equal(Uh, Uo)
    # odd grid: the cell at the origin exists and takes the floored source state
    assert np.isfinite(cp).all()


def test_solver_needs_a_gpu():
    if has_gpu():
        pytest.skip("a GPU is present")
    with pytest.raises(S.SetbError) as e:
        S.Solver(S.cart_desc(8))
    assert e.value.code == 8   # SETB_ENODEV: no CPU fallback


def test_slab_arguments_checked_on_the_host():
    """setb_init_slab validates the slab against the grid before touching a device."""
    from set_b200 import slab as SL
    desc = S.cart_desc((8, 6, 10))
    cp = np.zeros((8 * 6 * 4, 16))
    L = S.lib()
    h = C.c_void_p()
    for k0, n in ((0, 1), (-1, 4), (8, 4), (7, 4)):
        assert L.setb_init_slab(C.byref(h), C.byref(desc), k0, n, cp.ctypes.data_as(C.POINTER(C.c_double))) == 1
    if not has_gpu():
        assert L.setb_init_slab(C.byref(h), C.byref(desc), 2, 4, cp.ctypes.data_as(C.POINTER(C.c_double))) == 8
    assert SL.split_z(10, 3) == [(0, 4), (4, 3), (7, 3)]
    with pytest.raises(ValueError):
        SL.split_z(5, 3)
