"""Face-list grids: the reference's own geometry (cells + faces, Storage_module.f90:20-37).

`box_facelist` builds the face list of a (possibly stretched) box of hexahedral cells in the
reference's layouts and 1-based numbering -- Cell_center(3,N), Cell_Volume(N), Cell_gran(6,N),
Gran_normal(3,G), Gran_square(G), Gran_center(3,G), Gran_neighbour(2,G), Gran_neighbour_TVD(2,G),
Gran_type(G) -- optionally with cells and faces renumbered at random, so a caller can drive the
face-list path with grids that exercise arbitrary numbering and non-uniform spacing.
`FaceListSolver` is the device-resident solve on such a grid (setb_init_facelist).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import Solver, _check, _ip, _p, lib, lism_prim


class FlParams(C.Structure):
    _fields_ = [("r_src", C.c_double), ("rho_src", C.c_double), ("v_src", C.c_double),
                ("p_over_rho_src", C.c_double), ("r_floor", C.c_double), ("dt_init", C.c_double),
                ("face_skip_radius", C.c_double), ("cell_freeze_radius", C.c_double),
                ("physics", C.c_int32), ("powell", C.c_int32)]


def fl_params(r_src=0.125, rho_src=50.0, v_src=10.0, p_over_rho_src=0.01, r_floor=0.0, dt_init=2e-9,
              face_skip_radius=0.0, cell_freeze_radius=0.0, physics=0, powell=0) -> FlParams:
    """physics 0: conservative 3D ideal MHD; 1: the reference's axisymmetric hydro cell update
    with charge exchange against the H-atom fluids of Cell_par columns 9..16.  powell (physics 0):
    0 off, 1 the reference's div-B flux and momentum / induction sources, 2 plus the energy
    source."""
    p = FlParams()
    p.r_src, p.rho_src, p.v_src, p.p_over_rho_src, p.r_floor = r_src, rho_src, v_src, p_over_rho_src, r_floor
    p.dt_init, p.face_skip_radius, p.cell_freeze_radius = dt_init, face_skip_radius, cell_freeze_radius
    p.physics, p.powell = int(physics), int(powell)
    return p


@dataclass
class FaceList:
    """Arrays in the reference's Fortran layouts (row k of an [n, m] array is column k+1)."""
    cell_center: np.ndarray        # [N, 3] float64
    cell_volume: np.ndarray        # [N] float64
    cell_gran: np.ndarray          # [N, 6] int32, 1-based face numbers, 0 = none
    gran_normal: np.ndarray        # [G, 3] float64, unit, from neighbour 1 towards neighbour 2
    gran_square: np.ndarray        # [G] float64
    gran_center: np.ndarray        # [G, 3] float64
    gran_neighbour: np.ndarray     # [G, 2] int32, 1-based, -1 = none
    gran_neighbour_tvd: np.ndarray  # [G, 2] int32, 1-based, -1 = none
    gran_type: np.ndarray          # [G] int32

    @property
    def n_cell(self) -> int:
        return self.cell_volume.shape[0]

    @property
    def n_gran(self) -> int:
        return self.gran_square.shape[0]


# boundary face types of the six sides of a box (reference Gran_type: 2 = wall when the second
# neighbour is -1, 4 = outer boundary, 5 = axis)
DEFAULT_SIDES = {"x-": 4, "x+": 4, "y-": 5, "y+": 2, "z-": 2, "z+": 2}


def _nodes(n, lo, hi, stretch, rng):
    s = np.linspace(0.0, 1.0, n + 1)
    if stretch > 0.0:   # smooth monotone clustering towards the middle, plus seeded jitter
        s = s + stretch * np.sin(2.0 * np.pi * s) / (2.0 * np.pi)
        j = rng.uniform(-0.15, 0.15, n + 1) * stretch / n
        j[0] = j[-1] = 0.0
        s = np.sort(s + j)
    return lo + (hi - lo) * s


def box_facelist(shape, lo=(-1.0, -1.0, -1.0), hi=(1.0, 1.0, 1.0), stretch=0.0, sides=None,
                 permute_seed=None, seed=0) -> FaceList:
    """Face list of an nx x ny x nz box of hexahedra (node planes optionally stretched), with
    boundary faces typed per side and, when permute_seed is given, cells and faces renumbered by
    a seeded random permutation.  Neighbour 1 of an interior face is its low cell (normal along
    +axis); a boundary face's neighbour 1 is its cell, with the normal pointing out of the box."""
    nx, ny, nz = shape
    n = (nx, ny, nz)
    sides = dict(DEFAULT_SIDES, **(sides or {}))
    rng = np.random.default_rng(seed)
    xs = [_nodes(n[a], lo[a], hi[a], stretch, rng) for a in range(3)]
    ctr = [(x[1:] + x[:-1]) * 0.5 for x in xs]
    wid = [x[1:] - x[:-1] for x in xs]
    N = nx * ny * nz
    K, J, I = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    I, J, K = I.ravel(), J.ravel(), K.ravel()
    cell_center = np.stack([ctr[0][I], ctr[1][J], ctr[2][K]], -1)
    cell_volume = wid[0][I] * wid[1][J] * wid[2][K]

    def cnum(i, j, k):
        return i + nx * (j + ny * k)

    blocks = []
    cell_gran = np.zeros((N, 6), dtype=np.int64)
    G = 0
    for a in range(3):
        ext = list(n)
        ext[a] += 1
        Kf, Jf, If = np.meshgrid(np.arange(ext[2]), np.arange(ext[1]), np.arange(ext[0]), indexing="ij")
        idx = [If.ravel(), Jf.ravel(), Kf.ravel()]
        m = idx[a]
        cnt = m.size

        def shifted(d):
            t = [x.copy() for x in idx]
            t[a] = m + d
            ok = (t[a] >= 0) & (t[a] <= n[a] - 1)
            t[a] = np.clip(t[a], 0, n[a] - 1)
            return cnum(*t), ok

        low, has_low = shifted(-1)
        high, has_high = shifted(0)
        far_low, ok_fl = shifted(-2)
        far_high, ok_fh = shifted(1)
        interior = has_low & has_high
        s1 = np.where(has_low, low, high)
        s2 = np.where(interior, high, -1)
        ss1 = np.where(interior & ok_fl, far_low, -1)
        ss2 = np.where(interior & ok_fh, far_high, -1)
        nrm = np.zeros((cnt, 3))
        nrm[:, a] = np.where(has_low, 1.0, -1.0)
        o1, o2 = [b for b in range(3) if b != a]
        gc = np.zeros((cnt, 3))
        gc[:, a] = xs[a][m]
        gc[:, o1] = ctr[o1][idx[o1]]
        gc[:, o2] = ctr[o2][idx[o2]]
        sq = wid[o1][idx[o1]] * wid[o2][idx[o2]]
        ty = np.full(cnt, 2, dtype=np.int64)
        ty[~has_low] = sides["xyz"[a] + "-"]
        ty[~has_high] = sides["xyz"[a] + "+"]
        gid = G + np.arange(cnt)
        cell_gran[high[has_high], 2 * a] = gid[has_high]       # low face of the high cell
        cell_gran[low[has_low], 2 * a + 1] = gid[has_low]      # high face of the low cell
        blocks.append((nrm, sq, gc, np.stack([s1, s2], -1), np.stack([ss1, ss2], -1), ty))
        G += cnt
    gran_normal, gran_square, gran_center, nb, nbt, gtype = [np.concatenate(x) for x in zip(*blocks)]

    # renumbering: old cell c becomes cperm[c], old face g becomes fperm[g] (0-based)
    prng = np.random.default_rng(permute_seed) if permute_seed is not None else None
    cperm = prng.permutation(N) if prng is not None else np.arange(N)
    fperm = prng.permutation(G) if prng is not None else np.arange(G)
    cinv = np.argsort(cperm)
    finv = np.argsort(fperm)

    def remap(a):
        return np.where(a >= 0, cperm[np.maximum(a, 0)] + 1, -1)

    return FaceList(
        cell_center=np.ascontiguousarray(cell_center[cinv]),
        cell_volume=np.ascontiguousarray(cell_volume[cinv]),
        cell_gran=np.ascontiguousarray((fperm[cell_gran] + 1)[cinv].astype(np.int32)),
        gran_normal=np.ascontiguousarray(gran_normal[finv]),
        gran_square=np.ascontiguousarray(gran_square[finv]),
        gran_center=np.ascontiguousarray(gran_center[finv]),
        gran_neighbour=np.ascontiguousarray(remap(nb)[finv].astype(np.int32)),
        gran_neighbour_tvd=np.ascontiguousarray(remap(nbt)[finv].astype(np.int32)),
        gran_type=np.ascontiguousarray(gtype[finv].astype(np.int32)))


def lism_cellpar(mesh: FaceList, lism=None, seed=1, pert_amp=1e-3, params: FlParams | None = None) -> np.ndarray:
    """Seeded initial Cell_par [N,16] on a face list: the LISM state with +-pert_amp relative
    perturbations of rho and p (numpy generator keyed by seed), the source state inside r_src."""
    if lism is None:
        lism = lism_prim()
    N = mesh.n_cell
    rng = np.random.default_rng(seed)
    cp = np.zeros((N, 16))
    cp[:, :8] = np.asarray(lism, dtype=np.float64)
    cp[:, 0] *= 1.0 + pert_amp * rng.uniform(-1.0, 1.0, N)
    cp[:, 4] *= 1.0 + pert_amp * rng.uniform(-1.0, 1.0, N)
    if params is not None and params.r_src > 0.0:
        x = mesh.cell_center
        r = np.sqrt((x[:, 0] * x[:, 0] + x[:, 1] * x[:, 1]) + x[:, 2] * x[:, 2])
        m = r < params.r_src
        re = np.maximum(r[m], params.r_floor)
        rho = (params.r_src / re) ** 2 * params.rho_src
        cp[m, 0] = rho
        with np.errstate(invalid="ignore", divide="ignore"):
            for a in range(3):
                cp[m, 1 + a] = np.where(r[m] > 0.0, params.v_src * (x[m, a] / r[m]), 0.0)
        cp[m, 4] = params.p_over_rho_src * rho
        cp[m, 5:8] = 0.0
    return cp


class FaceListSolver(Solver):
    """A device-resident solve on a face list (setb_init_facelist); the state is indexed by the
    face list's cell numbers: conserved() returns U[8, N]."""

    def __init__(self, mesh: FaceList, cell_par: np.ndarray, params: FlParams):
        self.mesh = mesh
        self.N = mesh.n_cell
        self.shape = (self.N,)
        self.desc = None
        cp = np.ascontiguousarray(cell_par, dtype=np.float64)
        assert cp.shape == (self.N, 16)
        h = C.c_void_p()
        m = mesh
        i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32).ctypes.data_as(_ip)
        rc = lib().setb_init_facelist(C.byref(h), int(m.n_cell), int(m.n_gran), _p(cp), _p(m.cell_center),
                                      _p(m.cell_volume), i32(m.cell_gran), _p(m.gran_normal), _p(m.gran_square),
                                      _p(m.gran_center), i32(m.gran_neighbour), i32(m.gran_neighbour_tvd),
                                      i32(m.gran_type), C.byref(params))
        _check(rc, "setb_init_facelist")
        self.h = h


# ---------------------------------------------------------------------------- on-disk formats
def _i32p(a):
    return a.ctypes.data_as(_ip)


def read_fcmhd(path: str):
    """The reference's grid/state stream file (Set_Storage, Storage_module.f90:42-100): returns
    (time_all, cell_par [N,16], FaceList, gran_potok [G,9])."""
    t = C.c_double()
    n, g = C.c_int32(), C.c_int32()
    bpath = str(path).encode()
    _check(lib().setb_fcmhd_read_header(bpath, C.byref(t), C.byref(n), C.byref(g)), "setb_fcmhd_read_header")
    N, G = n.value, g.value
    cp = np.zeros((N, 16))
    m = FaceList(cell_center=np.zeros((N, 3)), cell_volume=np.zeros(N), cell_gran=np.zeros((N, 6), np.int32),
                 gran_normal=np.zeros((G, 3)), gran_square=np.zeros(G), gran_center=np.zeros((G, 3)),
                 gran_neighbour=np.zeros((G, 2), np.int32), gran_neighbour_tvd=np.zeros((G, 2), np.int32),
                 gran_type=np.zeros(G, np.int32))
    potok = np.zeros((G, 9))
    _check(lib().setb_fcmhd_read(bpath, N, G, C.byref(t), _p(cp), _p(m.cell_center), _p(m.cell_volume),
                                 _i32p(m.cell_gran), _p(m.gran_normal), _p(m.gran_square), _p(m.gran_center),
                                 _i32p(m.gran_neighbour), _i32p(m.gran_neighbour_tvd), _i32p(m.gran_type),
                                 _p(potok)), "setb_fcmhd_read")
    return t.value, cp, m, potok


def write_fcmhd(path: str, time_all: float, cell_par: np.ndarray, m: FaceList, gran_potok: np.ndarray | None = None):
    """Writes the grid/state stream file in the reference's format (zero fluxes when gran_potok
    is None, as the grid generator writes them)."""
    cp = np.ascontiguousarray(cell_par, dtype=np.float64)
    i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
    cg, nb, nbt, ty = i32(m.cell_gran), i32(m.gran_neighbour), i32(m.gran_neighbour_tvd), i32(m.gran_type)
    pot = None if gran_potok is None else np.ascontiguousarray(gran_potok, dtype=np.float64)
    _check(lib().setb_fcmhd_write(str(path).encode(), float(time_all), m.n_cell, m.n_gran, _p(cp), _p(m.cell_center),
                                  _p(m.cell_volume), _i32p(cg), _p(m.gran_normal), _p(m.gran_square),
                                  _p(m.gran_center), _i32p(nb), _i32p(nbt), _i32p(ty),
                                  _p(pot) if pot is not None else None), "setb_fcmhd_write")


def write_checkpoint(path: str, time_all: float, cell_par: np.ndarray):
    """Save_Storage (Storage_module.f90:160-182): time, Cell_par(16,N), 321.0."""
    cp = np.ascontiguousarray(cell_par, dtype=np.float64)
    _check(lib().setb_checkpoint_write(str(path).encode(), float(time_all), cp.shape[0], _p(cp)),
           "setb_checkpoint_write")


def read_checkpoint(path: str, n_cell: int):
    """Fill_data (Storage_module.f90:191-209): returns (time_all, cell_par [N,16])."""
    t = C.c_double()
    cp = np.zeros((n_cell, 16))
    _check(lib().setb_checkpoint_read(str(path).encode(), int(n_cell), C.byref(t), _p(cp)), "setb_checkpoint_read")
    return t.value, cp
