"""TEST INFRASTRUCTURE, NOT PRODUCT CODE.

ctypes front end of the CPU FP64 oracle (oracle/oracle.cpp), a restatement of SergeyMSU/SET's
MHD step (SET_Fortran_Cuda_MHD/Solvers.f90:1144-1859 chlld, :109-150 minmod/linear;
cuf_solvers.cuf:243-794 face/cell kernels; cuf_kernel.cuf:780-925 time loop) on a Cartesian
grid, plus the reference's own C++ Riemann solvers (SET_Gelios/source/Solvers.cpp: the HLL
HLLD_Solver_Alexashov :92-691, the HLLC HLLC_Aleksashov :1324-1639 and the HLLD HLLDQ_Korolkov
:1642-2185) built into oracle/_ref for pinning and cross-checks.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module.  The
product (set_b200) never does.

Parity status: chlld's shared set-up and HLL branch are pinned bit for bit against the compiled
reference C++ HLL solver, and its HLLC branch (B = 0) bit for bit against the reference's C++
HLLC; its HLLD branch is cross-checked to 1e-10 against the reference's second HLLD
(HLLDQ_Korolkov, axis-aligned faces).  The Cartesian and face-list drivers are restatements of
cuf_solvers.cuf checked by properties (the reference has no tests, and its Fortran path cannot be
compiled without a Fortran compiler).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(HERE, "liboracle.so")
_REF = os.path.join(HERE, "_ref", "libgelios_hll.so")
_lib = None
_ref = None

_dp = C.POINTER(C.c_double)


class OrcGrid(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("flags", C.c_int32),
                ("lo", C.c_double * 3), ("hi", C.c_double * 3), ("inflow", C.c_double * 8),
                ("r_src", C.c_double), ("rho_src", C.c_double), ("v_src", C.c_double),
                ("p_over_rho_src", C.c_double), ("r_floor", C.c_double), ("dt_init", C.c_double)]


class OrcOpts(C.Structure):
    _fields_ = [("n_state", C.c_int32), ("n_disc", C.c_int32), ("order", C.c_int32),
                ("scheme", C.c_int32), ("cfl", C.c_double)]


class OrcDiag(C.Structure):
    _fields_ = [("n_negdens", C.c_int64), ("first_bad_cell", C.c_int64), ("n_pfloor", C.c_int64),
                ("n_wave_err", C.c_int64), ("n_recon_err", C.c_int64), ("reserved", C.c_int64)]


class OrcClock(C.Structure):
    _fields_ = [("time_all", C.c_double), ("dt_next", C.c_double), ("dt_last", C.c_double)]


def build(force: bool = False) -> None:
    """Compile oracle/liboracle.so (and oracle/_ref when the reference tree is present)."""
    if force or not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(
            os.path.join(HERE, "oracle.cpp")):
        subprocess.check_call(["make", "-s", "-C", HERE], stdout=subprocess.DEVNULL)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        _lib = C.CDLL(_LIB)
        _lib.orc_chlld.restype = C.c_int
        _lib.orc_chlld.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, _dp, _dp,
                                   _dp, _dp, _dp, _dp, C.c_int]
        _lib.orc_chlld_q.restype = C.c_int
        _lib.orc_chlld_q.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, _dp, _dp,
                                     _dp, _dp, _dp, _dp, C.c_int, C.c_int, _dp]
        _lib.orc_minmod.restype = C.c_double
        _lib.orc_minmod.argtypes = [C.c_double, C.c_double]
        _lib.orc_linear.restype = C.c_double
        _lib.orc_linear.argtypes = [C.c_double] * 7
        _lib.orc_init_lism.argtypes = [C.POINTER(OrcGrid), _dp, C.c_uint64, C.c_double, _dp]
        _lib.orc_run.restype = C.c_int
        _lib.orc_run.argtypes = [C.POINTER(OrcGrid), C.POINTER(OrcOpts), _dp, C.POINTER(OrcClock),
                                 C.c_int, C.c_int, C.POINTER(OrcDiag)]
        _lib.orc_stage.argtypes = [C.POINTER(OrcGrid), C.POINTER(OrcOpts), _dp, _dp, _dp, C.c_double,
                                   C.c_int, _dp, C.c_int, C.POINTER(OrcDiag)]
        _lib.orc_clock_init.argtypes = [C.POINTER(OrcGrid), C.POINTER(OrcClock)]
        _lib.orc_prim_from_cons.argtypes = [_dp, _dp]
        _lib.orc_cons_from_prim.argtypes = [_dp, _dp]
        _lib.orc_cellpar_to_cons.argtypes = [C.c_int64, _dp, _dp]
        _lib.orc_cons_to_cellpar.argtypes = [C.c_int64, _dp, _dp]
        _lib.orc_max_threads.restype = C.c_int
    return _lib


def ref_available() -> bool:
    return os.path.exists(_REF)


def ref_lib():
    global _ref
    if _ref is None:
        _ref = C.CDLL(_REF)
        _ref.ref_gelios_hll.restype = C.c_double
        _ref.ref_gelios_hll.argtypes = [_dp, _dp, _dp, C.c_double, C.c_double, _dp, _dp, _dp, _dp]
        _ref.ref_gelios_hllc.restype = C.c_double
        _ref.ref_gelios_hllc.argtypes = [_dp, _dp, _dp, C.c_double, _dp]
        _ref.ref_korolkov.restype = C.c_double
        _ref.ref_korolkov.argtypes = [C.c_int, _dp, C.c_double, _dp, C.c_double, _dp, C.c_double, _dp, _dp]
    return _ref


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def chlld(n_state, normal, w, q1, q2, n_disc=0):
    """Scalar chlld: returns (status, qqq[8], dsl, dsp, dsc)."""
    q1 = np.ascontiguousarray(q1, dtype=np.float64)
    q2 = np.ascontiguousarray(q2, dtype=np.float64)
    out = np.zeros(8)
    dsl, dsp, dsc = C.c_double(), C.c_double(), C.c_double()
    rc = lib().orc_chlld(int(n_state), float(normal[0]), float(normal[1]), float(normal[2]), float(w),
                         _p(q1), _p(q2), C.byref(dsl), C.byref(dsp), C.byref(dsc), _p(out), int(n_disc))
    return rc, out, dsl.value, dsp.value, dsc.value


def chlld_q(n_state, normal, w, q1, q2, n_disc=0, ydar=False, konvect=None):
    """Scalar chlld_Q (Solvers.f90:198-1141): q1/q2 are 9-vectors (Q last).  konvect is None or
    (left, right) of the second passive scalar.  Returns (status, qqq[9], dsl, dsp, dsc, kflux)
    with kflux None when konvect is None."""
    q1 = np.ascontiguousarray(q1, dtype=np.float64)
    q2 = np.ascontiguousarray(q2, dtype=np.float64)
    assert q1.shape == (9,) and q2.shape == (9,)
    out = np.zeros(9)
    kv = None if konvect is None else np.array([konvect[0], konvect[1], 0.0])
    dsl, dsp, dsc = C.c_double(), C.c_double(), C.c_double()
    rc = lib().orc_chlld_q(int(n_state), float(normal[0]), float(normal[1]), float(normal[2]), float(w),
                           _p(q1), _p(q2), C.byref(dsl), C.byref(dsp), C.byref(dsc), _p(out), int(n_disc),
                           int(bool(ydar)), None if kv is None else _p(kv))
    return rc, out, dsl.value, dsp.value, dsc.value, (None if kv is None else kv[2])


def ref_hll(normal, w, q1, q2, dist=1.0):
    """The reference's own C++ HLL solver: returns (qqq[8], dsl, dsp, dsc)."""
    q1 = np.ascontiguousarray(q1, dtype=np.float64)
    q2 = np.ascontiguousarray(q2, dtype=np.float64)
    n = np.ascontiguousarray(normal, dtype=np.float64)
    out = np.zeros(8)
    dsl, dsp, dsc = C.c_double(), C.c_double(), C.c_double()
    ref_lib().ref_gelios_hll(_p(q1), _p(q2), _p(n), float(w), float(dist), _p(out), C.byref(dsl),
                             C.byref(dsp), C.byref(dsc))
    return out, dsl.value, dsp.value, dsc.value


def ref_hllc(normal, q1, q2):
    """The reference's own C++ HLLC solver (Solvers.cpp:1324-1639; B = 0, fixed face): returns the
    five fluxes (rho, mx, my, mz, E).  The B entries of q1/q2 are ignored."""
    q1 = np.ascontiguousarray(q1, dtype=np.float64)
    q2 = np.ascontiguousarray(q2, dtype=np.float64)
    n = np.ascontiguousarray(normal, dtype=np.float64)
    out = np.zeros(5)
    ref_lib().ref_gelios_hllc(_p(q1), _p(q2), _p(n), 1.0, _p(out))
    return out


def ref_korolkov(metod, normal, q1, q2, Q1=0.0, Q2=0.0):
    """The reference's HLLDQ_Korolkov (Solvers.cpp:1642-2185; metod 3 = HLLD, 2 = its HLLC
    variant) on an axis-aligned normal, w = 0: returns (qqq[8] in chlld's order, passive-scalar
    flux)."""
    q1 = np.ascontiguousarray(q1, dtype=np.float64)
    q2 = np.ascontiguousarray(q2, dtype=np.float64)
    n = np.ascontiguousarray(normal, dtype=np.float64)
    out = np.zeros(8)
    pq = C.c_double()
    ref_lib().ref_korolkov(int(metod), _p(q1), float(Q1), _p(q2), float(Q2), _p(n), 1.0, _p(out), C.byref(pq))
    return out, pq.value


def minmod(x, y):
    return lib().orc_minmod(float(x), float(y))


def linear(x1, t1, x2, t2, x3, t3, y):
    return lib().orc_linear(float(x1), float(t1), float(x2), float(t2), float(x3), float(t3), float(y))


def make_grid(n, lo=(-1.0, -1.0, -1.0), hi=(1.0, 1.0, 1.0), inflow=None, r_src=0.125, rho_src=50.0,
              v_src=10.0, p_over_rho_src=0.01, r_floor=0.0, dt_init=2e-9) -> OrcGrid:
    nx, ny, nz = (n, n, n) if np.isscalar(n) else n
    g = OrcGrid()
    g.nx, g.ny, g.nz, g.flags = int(nx), int(ny), int(nz), 0
    for a in range(3):
        g.lo[a] = lo[a]
        g.hi[a] = hi[a]
    if inflow is None:
        inflow = lism_prim()
    for v in range(8):
        g.inflow[v] = inflow[v]
    g.r_src, g.rho_src, g.v_src, g.p_over_rho_src, g.r_floor = r_src, rho_src, v_src, p_over_rho_src, r_floor
    g.dt_init = dt_init
    return g


def lism_prim(rho=1.0, p=1.0, u=(-2.0, 0.0, 0.0), bmag=1.0, tilt_deg=60.0):
    t = np.deg2rad(tilt_deg)
    return np.array([rho, u[0], u[1], u[2], p, bmag * np.cos(t), bmag * np.sin(t), 0.0])


def make_opts(n_state=3, order=2, scheme=2, cfl=0.4, n_disc=0) -> OrcOpts:
    o = OrcOpts()
    o.n_state, o.n_disc, o.order, o.scheme, o.cfl = n_state, n_disc, order, scheme, cfl
    return o


def init_lism(g: OrcGrid, lism=None, seed=1, pert_amp=1e-3) -> np.ndarray:
    """Conserved SoA state U[8, nz, ny, nx]."""
    if lism is None:
        lism = np.array(g.inflow[:])
    lism = np.ascontiguousarray(lism, dtype=np.float64)
    U = np.zeros((8, g.nz, g.ny, g.nx))
    lib().orc_init_lism(C.byref(g), _p(lism), C.c_uint64(seed), float(pert_amp), _p(U))
    return U


def clock_init(g: OrcGrid) -> OrcClock:
    ck = OrcClock()
    lib().orc_clock_init(C.byref(g), C.byref(ck))
    return ck


def run(g: OrcGrid, o: OrcOpts, U: np.ndarray, nsteps: int, clock: OrcClock | None = None, nthreads=0):
    """Advance U (conserved SoA, modified in place) by nsteps; returns (clock, diag)."""
    if clock is None:
        clock = clock_init(g)
    dg = OrcDiag()
    dg.first_bad_cell = -1
    lib().orc_run(C.byref(g), C.byref(o), _p(U), C.byref(clock), int(nsteps), int(nthreads), C.byref(dg))
    return clock, dg


def stage(g: OrcGrid, o: OrcOpts, Uin, dt, kind=0, Ubase=None, nthreads=0):
    """One stage: returns (Uout, dt_min, diag)."""
    Uout = np.zeros_like(Uin)
    dmin = C.c_double()
    dg = OrcDiag()
    dg.first_bad_cell = -1
    base = Ubase if Ubase is not None else Uin
    lib().orc_stage(C.byref(g), C.byref(o), _p(Uin), _p(base), _p(Uout), float(dt), int(kind),
                    C.byref(dmin), int(nthreads), C.byref(dg))
    return Uout, dmin.value, dg


def prim_from_cons(U8):
    U8 = np.ascontiguousarray(U8, dtype=np.float64)
    q = np.zeros(8)
    lib().orc_prim_from_cons(_p(U8), _p(q))
    return q


def cons_from_prim(q):
    q = np.ascontiguousarray(q, dtype=np.float64)
    U8 = np.zeros(8)
    lib().orc_cons_from_prim(_p(q), _p(U8))
    return U8


def cons_to_cellpar(U: np.ndarray) -> np.ndarray:
    """Conserved SoA -> Cell_par(16,N) (as a C array [N,16]); columns 9..16 zero."""
    N = U[0].size
    cp = np.zeros((N, 16))
    lib().orc_cons_to_cellpar(N, _p(np.ascontiguousarray(U)), _p(cp))
    return cp


def cellpar_to_cons(cp: np.ndarray, shape) -> np.ndarray:
    N = cp.shape[0]
    U = np.zeros((8,) + tuple(shape))
    lib().orc_cellpar_to_cons(N, _p(np.ascontiguousarray(cp)), _p(U))
    return U


def max_threads() -> int:
    return lib().orc_max_threads()


# ---------------------------------------------------------------------------- face-list grids
class OrcFaceList(C.Structure):
    _fields_ = [("n_cell", C.c_int64), ("n_gran", C.c_int64),
                ("cell_center", _dp), ("cell_volume", _dp), ("cell_gran", C.POINTER(C.c_int32)),
                ("gran_normal", _dp), ("gran_square", _dp), ("gran_center", _dp),
                ("gran_neighbour", C.POINTER(C.c_int32)), ("gran_neighbour_tvd", C.POINTER(C.c_int32)),
                ("gran_type", C.POINTER(C.c_int32)),
                ("r_src", C.c_double), ("rho_src", C.c_double), ("v_src", C.c_double),
                ("p_over_rho_src", C.c_double), ("r_floor", C.c_double), ("dt_init", C.c_double),
                ("face_skip_radius", C.c_double), ("cell_freeze_radius", C.c_double),
                ("hatom", _dp), ("physics", C.c_int32), ("powell", C.c_int32)]


def facelist(mesh, params, cell_par=None) -> OrcFaceList:
    """Oracle view of a face list (arrays in the reference's layouts, 1-based) and its
    parameters (anything with the fields of setb_fl_params); cell_par [N,16] supplies the H-atom
    fluids (columns 9..16) of physics 1.  Keep `mesh` and the returned object's `_keep` alive."""
    m = OrcFaceList()
    m.physics, m.powell = int(getattr(params, "physics", 0)), int(getattr(params, "powell", 0))
    if cell_par is not None:
        h = np.ascontiguousarray(np.asarray(cell_par, dtype=np.float64)[:, 8:16])
        m.hatom = _p(h)
        m._keep = h
    m.n_cell, m.n_gran = mesh.n_cell, mesh.n_gran
    i32 = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
    m.cell_center, m.cell_volume, m.cell_gran = _p(mesh.cell_center), _p(mesh.cell_volume), i32(mesh.cell_gran)
    m.gran_normal, m.gran_square, m.gran_center = _p(mesh.gran_normal), _p(mesh.gran_square), _p(mesh.gran_center)
    m.gran_neighbour, m.gran_neighbour_tvd, m.gran_type = (i32(mesh.gran_neighbour), i32(mesh.gran_neighbour_tvd),
                                                          i32(mesh.gran_type))
    for f in ("r_src", "rho_src", "v_src", "p_over_rho_src", "r_floor", "dt_init", "face_skip_radius",
              "cell_freeze_radius"):
        setattr(m, f, float(getattr(params, f)))
    return m


def fl_run(m: OrcFaceList, o: OrcOpts, U: np.ndarray, nsteps: int, clock: OrcClock | None = None,
           flux: np.ndarray | None = None, nthreads=0):
    """Advance the face-list state U[8, N] (conserved, modified in place) by nsteps with the
    persistent face flux array `flux` [G, 9] (zeros when None).  Returns (clock, diag, flux)."""
    if clock is None:
        clock = OrcClock()
        clock.time_all, clock.dt_next, clock.dt_last = 0.0, m.dt_init, 0.0
    if flux is None:
        flux = np.zeros((m.n_gran, 9))
    dg = OrcDiag()
    dg.first_bad_cell = -1
    lib().orc_fl_run(C.byref(m), C.byref(o), _p(U), _p(flux), C.byref(clock), int(nsteps), int(nthreads),
                     C.byref(dg))
    return clock, dg, flux
