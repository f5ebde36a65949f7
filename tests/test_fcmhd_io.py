"""The reference's on-disk formats through the C ABI (setb_fcmhd_* / setb_checkpoint_*): round
trips, the byte layout of Set_Storage / Save_Storage (Storage_module.f90:42-209) built here
independently with numpy, and rejection of damaged files."""
import ctypes as C

import numpy as np
import pytest

import set_b200 as S
from set_b200 import facelist as FL


def sample(seed=0):
    m = FL.box_facelist((5, 4, 3), stretch=0.4, permute_seed=seed + 1, seed=seed)
    rng = np.random.default_rng(seed)
    cp = rng.uniform(0.1, 2.0, (m.n_cell, 16))
    pot = rng.normal(size=(m.n_gran, 9))
    return m, cp, pot


def expected_bytes(t, cp, m, pot):
    f64 = lambda a: np.ascontiguousarray(a, dtype="<f8").tobytes()
    i32 = lambda a: np.ascontiguousarray(a, dtype="<i4").tobytes()
    return b"".join([f64(t), i32(m.n_cell), i32(m.n_gran), f64(cp), f64(m.cell_center), f64(m.cell_volume),
                     i32(m.cell_gran), f64(m.gran_normal), f64(m.gran_square), f64(m.gran_center),
                     i32(m.gran_neighbour), i32(m.gran_neighbour_tvd), f64(121.0), i32(m.gran_type), f64(122.0),
                     f64(pot), f64(123.0)])


def test_grid_file_round_trip_and_byte_layout(tmp_path):
    m, cp, pot = sample()
    p = tmp_path / "FCMHD_3.bin"
    FL.write_fcmhd(p, 12.5, cp, m, pot)
    assert p.read_bytes() == expected_bytes(12.5, cp, m, pot)
    t, cp2, m2, pot2 = FL.read_fcmhd(p)
    assert t == 12.5 and np.array_equal(cp2, cp) and np.array_equal(pot2, pot)
    for k in m.__dataclass_fields__:
        assert np.array_equal(getattr(m2, k), getattr(m, k)), k
    # zero fluxes when none are given, as the grid generator writes them
    FL.write_fcmhd(p, 0.0, cp, m)
    assert not FL.read_fcmhd(p)[3].any()


def test_grid_file_damage_is_rejected(tmp_path):
    m, cp, pot = sample(2)
    good = expected_bytes(1.0, cp, m, pot)
    p = tmp_path / "g.bin"
    cases = {
        "truncated": good[:-5],
        "trailing": good + b"\0",
        "sentinel121": good.replace(np.float64(121.0).tobytes(), np.float64(120.0).tobytes()),
        "sentinel123": good[:-8] + np.float64(124.0).tobytes(),
    }
    for name, data in cases.items():
        p.write_bytes(data)
        with pytest.raises(S.SetbError) as e:
            FL.read_fcmhd(p)
        assert e.value.code == 10, name
    # counts that differ from the caller's buffers
    p.write_bytes(good)
    buf = lambda n: np.zeros(n)
    ib = lambda n: np.zeros(n, np.int32).ctypes.data_as(S._ip)
    N, G = m.n_cell, m.n_gran
    t = C.c_double()
    rc = S.lib().setb_fcmhd_read(str(p).encode(), N - 1, G, C.byref(t), S._p(buf(16 * N)), S._p(buf(3 * N)),
                                 S._p(buf(N)), ib(6 * N), S._p(buf(3 * G)), S._p(buf(G)), S._p(buf(3 * G)),
                                 ib(2 * G), ib(2 * G), ib(G), None)
    assert rc == 10
    with pytest.raises(S.SetbError) as e:
        FL.read_fcmhd(tmp_path / "missing.bin")
    assert e.value.code == 10


def test_checkpoint_round_trip_and_layout(tmp_path):
    rng = np.random.default_rng(4)
    cp = rng.normal(size=(37, 16))
    p = tmp_path / "FCMHD_3.5_out.bin"
    FL.write_checkpoint(p, 3.25, cp)
    assert p.read_bytes() == np.float64(3.25).tobytes() + cp.astype("<f8").tobytes() + np.float64(321.0).tobytes()
    t, cp2 = FL.read_checkpoint(p, 37)
    assert t == 3.25 and np.array_equal(cp2, cp)
    with pytest.raises(S.SetbError):
        FL.read_checkpoint(p, 36)          # wrong cell count: the sentinel is not where expected
    p.write_bytes(p.read_bytes()[:-8] + np.float64(320.0).tobytes())
    with pytest.raises(S.SetbError):
        FL.read_checkpoint(p, 37)
