"""set_b200 -- B200-native ideal-MHD finite-volume step (SergeyMSU/SET FCMHD hot path).

Python front end over the C ABI of libsetb200.so (include/setb200.h).  The names mirror the
reference's solver-module interface:

    chlld(...)                  Solvers.f90:1144-1859 (host), chlld_batch(...) on the GPU
    chlld_q(...)                Solvers.f90:198-1141 (host), chlld_q_batch(...) on the GPU
    Solver.init_cartesian(...)  Set_CUDA (cuf_kernel.cuf:351-382)
    Solver.step(n, opts)        the CUDA_START_MGD time loop (cuf_kernel.cuf:780-925)
    Solver.get_state()          Send_data_to_Host (cuf_kernel.cuf:384-400)
    Solver.set_state(cp, t)     Fill_data restart (Storage_module.f90:191-209)

There is no CPU fallback: every call goes through the compiled CUDA library, and importing a
function that needs it raises if libsetb200.so has not been built
(``python -m set_b200.build``).
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libsetb200.so")

SETB_OK = 0
ERRORS = {
    1: "EINVAL", 2: "ECUDA", 3: "ENOMEM", 4: "ENEGDENS", 5: "EWAVES", 6: "ERECON", 7: "ETIMEOUT",
    8: "ENODEV", 9: "ESIZE", 10: "EIO", 11: "EBUSY",
}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class SetbError(RuntimeError):
    def __init__(self, code: int, where: str):
        self.code = code
        super().__init__(f"{where}: {ERRORS.get(code, code)} ({lib().setb_strerror(code).decode()})")


class CartDesc(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("flags", C.c_int32),
                ("lo", C.c_double * 3), ("hi", C.c_double * 3), ("inflow", C.c_double * 8),
                ("r_src", C.c_double), ("rho_src", C.c_double), ("v_src", C.c_double),
                ("p_over_rho_src", C.c_double), ("r_floor", C.c_double), ("dt_init", C.c_double)]


class LismIC(C.Structure):
    _fields_ = [("lism", C.c_double * 8), ("seed", C.c_uint64), ("pert_amp", C.c_double)]


class StepOpts(C.Structure):
    _fields_ = [("n_state", C.c_int32), ("n_disc", C.c_int32), ("order", C.c_int32),
                ("scheme", C.c_int32), ("precision", C.c_int32), ("reserved", C.c_int32),
                ("cfl", C.c_double)]


class Diag(C.Structure):
    _fields_ = [("time_all", C.c_double), ("dt_next", C.c_double), ("dt_last", C.c_double),
                ("steps", C.c_int64), ("n_negdens", C.c_int64), ("first_bad_cell", C.c_int64),
                ("n_pfloor", C.c_int64), ("n_wave_err", C.c_int64), ("n_recon_err", C.c_int64),
                ("n_fp64_redo", C.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Request(C.Structure):
    _fields_ = [("desc", CartDesc), ("ic", LismIC), ("opts", StepOpts), ("max_steps", C.c_int32),
                ("reserved", C.c_int32), ("steady_tol", C.c_double), ("result_U", _dp)]


class Result(C.Structure):
    _fields_ = [("id", C.c_int64), ("status", C.c_int32), ("steps", C.c_int32), ("converged", C.c_int32),
                ("reserved", C.c_int32), ("last_change", C.c_double), ("time_all", C.c_double),
                ("t_submit", C.c_double), ("t_admit", C.c_double), ("t_done", C.c_double), ("diag", Diag)]


# Every entry point of include/setb200.h: name -> (restype, argtypes)
_SIGS = {
    "setb_version": (C.c_int32, []),
    "setb_strerror": (C.c_char_p, [C.c_int32]),
    "setb_chlld": (C.c_int32, [_ip, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _ip]),
    "setb_chlld_batch": (C.c_int32, [C.c_int64, C.c_int32, C.c_int32, C.c_int32, _dp, _dp, _dp, _dp,
                                     _dp, _dp, _ip]),
    "setb_chlld_q": (C.c_int32, [_ip, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _ip, _ip, _ip, _dp, _ip]),
    "setb_chlld_q_batch": (C.c_int32, [C.c_int64, C.c_int32, C.c_int32, C.c_int32, _dp, _dp, _dp, _dp, _dp,
                                       _dp, _dp, _ip]),
    "setb_init_cartesian": (C.c_int32, [C.POINTER(C.c_void_p), C.POINTER(CartDesc), _dp]),
    "setb_init_cartesian_lism": (C.c_int32, [C.POINTER(C.c_void_p), C.POINTER(CartDesc), C.POINTER(LismIC)]),
    "setb_cart_fill_lism": (C.c_int32, [C.POINTER(CartDesc), C.POINTER(LismIC), _dp]),
    "setb_step": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(StepOpts), _dp]),
    "setb_step_profiled": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(StepOpts), _dp, _dp, _ip]),
    "setb_sync": (C.c_int32, [C.c_void_p]),
    "setb_get_state": (C.c_int32, [C.c_void_p, _dp, _dp]),
    "setb_set_state": (C.c_int32, [C.c_void_p, _dp, C.c_double]),
    "setb_state_view": (C.c_int32, [C.c_void_p, C.POINTER(_dp), C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                    C.POINTER(C.c_int64)]),
    "setb_get_conserved": (C.c_int32, [C.c_void_p, _dp]),
    "setb_copy_state": (C.c_int32, [C.c_void_p, C.c_void_p]),
    "setb_status": (C.c_int32, [C.c_void_p, C.POINTER(Diag)]),
    "setb_stream": (C.c_int32, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "setb_set_copy_wait": (C.c_int32, [C.c_void_p, C.c_int64]),
    "setb_init_slab": (C.c_int32, [C.POINTER(C.c_void_p), C.POINTER(CartDesc), C.c_int32, C.c_int32, _dp]),
    "setb_slab_stage": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(StepOpts)]),
    "setb_slab_view": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(_dp), C.POINTER(C.c_int64),
                                   C.POINTER(C.c_int64), _ip]),
    "setb_slab_dt": (C.c_int32, [C.c_void_p, C.POINTER(_dp)]),
    "setb_destroy": (C.c_int32, [C.c_void_p]),
    "setb_step_noalloc": (C.c_int32, [C.POINTER(CartDesc), C.POINTER(StepOpts), C.c_void_p, C.c_int64, C.c_int32,
                                      _dp, _dp, C.POINTER(Diag), C.c_void_p]),
    "setb_init_facelist": (C.c_int32, [C.POINTER(C.c_void_p), C.c_int32, C.c_int32, _dp, _dp, _dp, _ip, _dp, _dp,
                                       _dp, _ip, _ip, _ip, C.c_void_p]),
    "setb_fcmhd_read_header": (C.c_int32, [C.c_char_p, _dp, _ip, _ip]),
    "setb_fcmhd_read": (C.c_int32, [C.c_char_p, C.c_int32, C.c_int32, _dp, _dp, _dp, _dp, _ip, _dp, _dp, _dp, _ip,
                                    _ip, _ip, _dp]),
    "setb_fcmhd_write": (C.c_int32, [C.c_char_p, C.c_double, C.c_int32, C.c_int32, _dp, _dp, _dp, _ip, _dp, _dp,
                                     _dp, _ip, _ip, _ip, _dp]),
    "setb_checkpoint_write": (C.c_int32, [C.c_char_p, C.c_double, C.c_int32, _dp]),
    "setb_checkpoint_read": (C.c_int32, [C.c_char_p, C.c_int32, _dp, _dp]),
    "setb_batch_create": (C.c_int32, [C.POINTER(C.c_void_p), C.c_int32, C.c_int32, C.c_int64]),
    "setb_batch_add": (C.c_int32, [C.c_void_p, C.POINTER(CartDesc), C.POINTER(LismIC), C.POINTER(StepOpts), _ip]),
    "setb_batch_remove": (C.c_int32, [C.c_void_p, C.c_int32]),
    "setb_batch_step": (C.c_int32, [C.c_void_p, C.c_int32]),
    "setb_batch_check": (C.c_int32, [C.c_void_p, _dp]),
    "setb_batch_get_conserved": (C.c_int32, [C.c_void_p, C.c_int32, _dp]),
    "setb_batch_status": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(Diag)]),
    "setb_batch_info": (C.c_int32, [C.c_void_p, C.POINTER(C.c_int64), _ip, _ip, _ip]),
    "setb_batch_set_tiling": (C.c_int32, [C.c_void_p, C.c_int32, C.c_int32]),
    "setb_batch_tune": (C.c_int32, [C.c_void_p, C.c_int32, _ip, _ip, _dp]),
    "setb_batch_sync": (C.c_int32, [C.c_void_p]),
    "setb_batch_destroy": (C.c_int32, [C.c_void_p]),
    "setb_server_create": (C.c_int32, [C.POINTER(C.c_void_p), C.c_int32, C.c_int32, C.c_int64, C.c_int32]),
    "setb_server_submit": (C.c_int32, [C.c_void_p, C.POINTER(Request), C.POINTER(C.c_int64)]),
    "setb_server_wait": (C.c_int32, [C.c_void_p, C.c_int64, C.POINTER(Result), C.c_double]),
    "setb_server_poll": (C.c_int32, [C.c_void_p, C.POINTER(Result), C.c_int32, _ip]),
    "setb_server_stats": (C.c_int32, [C.c_void_p, _ip, _ip, C.POINTER(C.c_int64), C.POINTER(C.c_int64), _ip]),
    "setb_server_destroy": (C.c_int32, [C.c_void_p]),
}

_lib = None


def lib():
    """The loaded libsetb200.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m set_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(rc: int, where: str):
    if rc != SETB_OK:
        raise SetbError(rc, where)


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous, "need a C-contiguous float64 array"
    return a.ctypes.data_as(_dp)


# ------------------------------------------------------------------------ problem builders
def lism_prim(rho=1.0, p=1.0, u=(-2.0, 0.0, 0.0), bmag=1.0, tilt_deg=60.0) -> np.ndarray:
    """LISM primitive state (rho,u,v,w,p,Bx,By,Bz); B in the reference's stored units, tilted
    tilt_deg from x in the x-y plane."""
    t = math.radians(tilt_deg)
    return np.array([rho, u[0], u[1], u[2], p, bmag * math.cos(t), bmag * math.sin(t), 0.0])


def cart_desc(n, lo=(-1.0, -1.0, -1.0), hi=(1.0, 1.0, 1.0), inflow=None, r_src=0.125, rho_src=50.0,
              v_src=10.0, p_over_rho_src=0.01, r_floor=None, dt_init=2e-9) -> CartDesc:
    """Cartesian problem: LISM inflow at x = hi, zero-gradient elsewhere, solar-wind source
    inside r_src.  r_floor defaults to half the smallest cell size, which only affects a cell
    centred at the origin (odd grids)."""
    nx, ny, nz = (n, n, n) if np.isscalar(n) else n
    d = CartDesc()
    d.nx, d.ny, d.nz, d.flags = int(nx), int(ny), int(nz), 0
    for a in range(3):
        d.lo[a], d.hi[a] = lo[a], hi[a]
    if inflow is None:
        inflow = lism_prim()
    for v in range(8):
        d.inflow[v] = float(inflow[v])
    if r_floor is None:
        r_floor = 0.5 * min((hi[a] - lo[a]) / m for a, m in enumerate((nx, ny, nz)))
    d.r_src, d.rho_src, d.v_src, d.p_over_rho_src, d.r_floor = r_src, rho_src, v_src, p_over_rho_src, r_floor
    d.dt_init = dt_init
    return d


def lism_ic(lism=None, seed=1, pert_amp=1e-3) -> LismIC:
    ic = LismIC()
    if lism is None:
        lism = lism_prim()
    for v in range(8):
        ic.lism[v] = float(lism[v])
    ic.seed = int(seed)
    ic.pert_amp = float(pert_amp)
    return ic


def step_opts(n_state=3, order=2, scheme=2, cfl=0.4, n_disc=0, precision=0) -> StepOpts:
    o = StepOpts()
    o.n_state, o.n_disc, o.order, o.scheme, o.precision, o.reserved = n_state, n_disc, order, scheme, precision, 0
    o.cfl = cfl
    return o


def fill_lism(desc: CartDesc, ic: LismIC) -> np.ndarray:
    """Host generator of the seeded initial condition as Cell_par, returned as an [N,16] array
    (row c = Fortran column c+1)."""
    N = desc.nx * desc.ny * desc.nz
    cp = np.zeros((N, 16))
    _check(lib().setb_cart_fill_lism(C.byref(desc), C.byref(ic), _p(cp)), "setb_cart_fill_lism")
    return cp


# ------------------------------------------------------------------------ flux routine
def chlld(n_state, normal, w, qqq1, qqq2, n_disc=None):
    """The reference's chlld signature on the host: returns (qqq[8], dsl, dsp, dsc)."""
    q1 = np.ascontiguousarray(qqq1, dtype=np.float64)
    q2 = np.ascontiguousarray(qqq2, dtype=np.float64)
    out = np.zeros(8)
    ns = C.c_int32(int(n_state))
    al, be, ge, wv = (C.c_double(float(normal[0])), C.c_double(float(normal[1])),
                      C.c_double(float(normal[2])), C.c_double(float(w)))
    dsl, dsp, dsc = C.c_double(), C.c_double(), C.c_double()
    nd = C.byref(C.c_int32(int(n_disc))) if n_disc is not None else None
    rc = lib().setb_chlld(C.byref(ns), C.byref(al), C.byref(be), C.byref(ge), C.byref(wv), _p(q1), _p(q2),
                          C.byref(dsl), C.byref(dsp), C.byref(dsc), _p(out), nd)
    _check(rc, "setb_chlld")
    return out, dsl.value, dsp.value, dsc.value


def chlld_batch(n_state, normals, q1, q2, w=None, n_disc=0, precision=0):
    """Batched chlld on the GPU.  normals [n,3], q1/q2 [n,8] primitive states.
    Returns (qqq [n,8], speeds [n,3] = (dsl, dsp, dsc), flags [n])."""
    normals = np.ascontiguousarray(normals, dtype=np.float64)
    q1 = np.ascontiguousarray(q1, dtype=np.float64)
    q2 = np.ascontiguousarray(q2, dtype=np.float64)
    n = q1.shape[0]
    qqq = np.zeros((n, 8))
    sp = np.zeros((n, 3))
    fl = np.zeros(n, dtype=np.int32)
    wp = _p(np.ascontiguousarray(w, dtype=np.float64)) if w is not None else None
    rc = lib().setb_chlld_batch(n, int(n_state), int(n_disc), int(precision), _p(normals), wp, _p(q1), _p(q2),
                                _p(qqq), _p(sp), fl.ctypes.data_as(_ip))
    _check(rc, "setb_chlld_batch")
    return qqq, sp, fl


def chlld_q(n_state, normal, w, qqq1, qqq2, n_disc=None, ydar=None, konvect=None, null_bn=None,
            p_correct=None):
    """The reference's chlld_Q signature on the host (Solvers.f90:198-201).  qqq1 / qqq2 are
    9-vectors (Q last); konvect is None or (left, right) of the second scalar; the logical
    OPTIONAL arguments are None (absent) or bools.  Returns (qqq[9], dsl, dsp, dsc, kflux) with
    kflux None when konvect is None."""
    q1 = np.ascontiguousarray(qqq1, dtype=np.float64)
    q2 = np.ascontiguousarray(qqq2, dtype=np.float64)
    if q1.shape != (9,) or q2.shape != (9,):
        raise ValueError("chlld_q takes 9-component states")
    out = np.zeros(9)
    ns = C.c_int32(int(n_state))
    al, be, ge, wv = (C.c_double(float(normal[0])), C.c_double(float(normal[1])),
                      C.c_double(float(normal[2])), C.c_double(float(w)))
    dsl, dsp, dsc = C.c_double(), C.c_double(), C.c_double()
    opt = lambda v: C.byref(C.c_int32(int(v))) if v is not None else None
    kv = np.array([konvect[0], konvect[1], 0.0]) if konvect is not None else None
    rc = lib().setb_chlld_q(C.byref(ns), C.byref(al), C.byref(be), C.byref(ge), C.byref(wv), _p(q1), _p(q2),
                            C.byref(dsl), C.byref(dsp), C.byref(dsc), _p(out), opt(null_bn), opt(n_disc),
                            opt(p_correct), _p(kv) if kv is not None else None, opt(ydar))
    _check(rc, "setb_chlld_q")
    return out, dsl.value, dsp.value, dsc.value, (None if kv is None else kv[2])


def chlld_q_batch(n_state, normals, q1, q2, w=None, n_disc=0, ydar=False, konvect=None):
    """Batched chlld_Q on the GPU.  normals [n,3], q1/q2 [n,9]; konvect None or [n,2] (left,
    right).  Returns (qqq [n,9], speeds [n,3], flags [n], kflux [n] or None)."""
    normals = np.ascontiguousarray(normals, dtype=np.float64)
    q1 = np.ascontiguousarray(q1, dtype=np.float64)
    q2 = np.ascontiguousarray(q2, dtype=np.float64)
    n = q1.shape[0]
    qqq = np.zeros((n, 9))
    sp = np.zeros((n, 3))
    fl = np.zeros(n, dtype=np.int32)
    kv = None
    if konvect is not None:
        kv = np.zeros((n, 3))
        kv[:, :2] = konvect
    wp = _p(np.ascontiguousarray(w, dtype=np.float64)) if w is not None else None
    rc = lib().setb_chlld_q_batch(n, int(n_state), int(n_disc), int(bool(ydar)), _p(normals), wp, _p(q1), _p(q2),
                                  _p(kv) if kv is not None else None, _p(qqq), _p(sp), fl.ctypes.data_as(_ip))
    _check(rc, "setb_chlld_q_batch")
    return qqq, sp, fl, (None if kv is None else kv[:, 2].copy())


def step_noalloc(desc: CartDesc, opts: StepOpts, U_ptr: int, var_stride: int, nsteps: int, dt: float,
                 time_all: float, stream: int = 0):
    """setb_step_noalloc: advance a caller-owned device state (8 planes at var_stride) in place
    without any allocation by the library.  Returns (dt for the next step, time, Diag)."""
    dt_c, t_c = C.c_double(dt), C.c_double(time_all)
    d = Diag()
    rc = lib().setb_step_noalloc(C.byref(desc), C.byref(opts), C.c_void_p(U_ptr), int(var_stride), int(nsteps),
                                 C.byref(dt_c), C.byref(t_c), C.byref(d), C.c_void_p(stream or None))
    _check(rc, "setb_step_noalloc")
    return dt_c.value, t_c.value, d


# ------------------------------------------------------------------------ device-resident solver
class Solver:
    """A device-resident Cartesian solve (one handle, one CUDA stream)."""

    def __init__(self, desc: CartDesc, cell_par: np.ndarray | None = None, ic: LismIC | None = None):
        self.desc = desc
        self.shape = (desc.nz, desc.ny, desc.nx)
        self.N = desc.nx * desc.ny * desc.nz
        h = C.c_void_p()
        if cell_par is not None:
            cp = np.ascontiguousarray(cell_par, dtype=np.float64)
            assert cp.shape == (self.N, 16)
            _check(lib().setb_init_cartesian(C.byref(h), C.byref(desc), _p(cp)), "setb_init_cartesian")
        else:
            _check(lib().setb_init_cartesian_lism(C.byref(h), C.byref(desc), C.byref(ic or lism_ic())),
                   "setb_init_cartesian_lism")
        self.h = h

    def close(self):
        if self.h:
            lib().setb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def step(self, nsteps: int, opts: StepOpts, wait: bool = True, check: bool = True):
        """Advance nsteps; returns the simulated time when wait, else None (asynchronous)."""
        t = C.c_double()
        rc = lib().setb_step(self.h, int(nsteps), C.byref(opts), C.byref(t) if wait else None)
        if check:
            _check(rc, "setb_step")
        return t.value if wait else rc

    def step_profiled(self, nsteps: int, opts: StepOpts):
        """Advance nsteps timing every kernel with CUDA events on the handle's stream.
        Returns (time_all, [ms stage-1 kernels, ms stage-2 kernels], [launch counts])."""
        t = C.c_double()
        ms = (C.c_double * 2)()
        n = (C.c_int32 * 2)()
        _check(lib().setb_step_profiled(self.h, int(nsteps), C.byref(opts), C.byref(t), ms, n),
               "setb_step_profiled")
        return t.value, [ms[0], ms[1]], [n[0], n[1]]

    def sync(self) -> int:
        return lib().setb_sync(self.h)

    def get_state(self, out: np.ndarray | None = None):
        """Cell_par [N,16] (columns 9..16 of `out` untouched) and the simulated time."""
        if out is None:
            out = np.zeros((self.N, 16))
        t = C.c_double()
        _check(lib().setb_get_state(self.h, _p(out), C.byref(t)), "setb_get_state")
        return out, t.value

    def set_state(self, cell_par: np.ndarray, time_all: float = 0.0):
        cp = np.ascontiguousarray(cell_par, dtype=np.float64)
        _check(lib().setb_set_state(self.h, _p(cp), float(time_all)), "setb_set_state")

    def status(self) -> Diag:
        d = Diag()
        _check(lib().setb_status(self.h, C.byref(d)), "setb_status")
        return d

    def state_view(self):
        """(device pointer, var_stride, plane_stride, row_pitch) of the conserved SoA state."""
        base = _dp()
        vs, ps, px = C.c_int64(), C.c_int64(), C.c_int64()
        _check(lib().setb_state_view(self.h, C.byref(base), C.byref(vs), C.byref(ps), C.byref(px)),
               "setb_state_view")
        return C.cast(base, C.c_void_p).value, vs.value, ps.value, px.value

    def copy_from(self, other: "Solver"):
        """Device-side copy of another handle's state, clock and counters (same grid)."""
        _check(lib().setb_copy_state(self.h, other.h), "setb_copy_state")

    def set_copy_wait(self, cycles: int):
        """Limit of the stage kernels' first wait on a plane copy (SM cycles; 0 = default ~2 s,
        < 0 = one non-blocking check)."""
        _check(lib().setb_set_copy_wait(self.h, int(cycles)), "setb_set_copy_wait")

    def stream(self) -> int:
        s = C.c_void_p()
        _check(lib().setb_stream(self.h, C.byref(s)), "setb_stream")
        return s.value or 0

    def conserved(self) -> np.ndarray:
        """Conserved state U[8, nz, ny, nx] (rho, mx, my, mz, E, Bx, By, Bz) on the host."""
        U = np.zeros((8,) + self.shape)
        _check(lib().setb_get_conserved(self.h, _p(U)), "setb_get_conserved")
        return U


@dataclass
class Problem:
    """A named problem: grid + initial condition + scheme."""
    desc: CartDesc
    ic: LismIC
    opts: StepOpts
    steps: int


class Batch:
    """Many Cartesian solves advanced together (setb_batch_*): admission by HBM footprint,
    add/remove between steps, per-solve lagged dt."""

    def __init__(self, max_slots: int, precision: int = 1, hbm_budget: int = 150 * 10 ** 9):
        h = C.c_void_p()
        _check(lib().setb_batch_create(C.byref(h), int(max_slots), int(precision), int(hbm_budget)),
               "setb_batch_create")
        self.h = h
        self.max_slots = max_slots
        self.precision = precision
        self.shapes = {}

    def close(self):
        if self.h:
            lib().setb_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def add(self, desc: CartDesc, ic: LismIC, opts: StepOpts) -> int:
        """Admit a solve; returns its slot, or raises SetbError(EBUSY=11) when it does not fit."""
        slot = C.c_int32()
        _check(lib().setb_batch_add(self.h, C.byref(desc), C.byref(ic), C.byref(opts), C.byref(slot)),
               "setb_batch_add")
        self.shapes[slot.value] = (desc.nz, desc.ny, desc.nx)
        return slot.value

    def try_add(self, desc: CartDesc, ic: LismIC, opts: StepOpts):
        """Admit a solve; None when it does not fit (budget or slots)."""
        slot = C.c_int32()
        rc = lib().setb_batch_add(self.h, C.byref(desc), C.byref(ic), C.byref(opts), C.byref(slot))
        if rc == 11:
            return None
        _check(rc, "setb_batch_add")
        self.shapes[slot.value] = (desc.nz, desc.ny, desc.nx)
        return slot.value

    def remove(self, slot: int):
        _check(lib().setb_batch_remove(self.h, int(slot)), "setb_batch_remove")
        self.shapes.pop(slot, None)

    def step(self, nsteps: int):
        _check(lib().setb_batch_step(self.h, int(nsteps)), "setb_batch_step")

    def sync(self):
        _check(lib().setb_batch_sync(self.h), "setb_batch_sync")

    def check(self) -> np.ndarray:
        out = np.zeros(self.max_slots)
        _check(lib().setb_batch_check(self.h, _p(out)), "setb_batch_check")
        return out

    def conserved(self, slot: int) -> np.ndarray:
        U = np.zeros((8,) + self.shapes[slot])
        _check(lib().setb_batch_get_conserved(self.h, int(slot), _p(U)), "setb_batch_get_conserved")
        return U

    def status(self, slot: int, check: bool = True) -> Diag:
        d = Diag()
        rc = lib().setb_batch_status(self.h, int(slot), C.byref(d))
        if check:
            _check(rc, "setb_batch_status")
        return d

    def info(self):
        used, act, lz, grid = C.c_int64(), C.c_int32(), C.c_int32(), C.c_int32()
        _check(lib().setb_batch_info(self.h, C.byref(used), C.byref(act), C.byref(lz), C.byref(grid)),
               "setb_batch_info")
        return {"bytes_used": used.value, "active": act.value, "lz": lz.value, "grid": grid.value}

    def set_tiling(self, lz: int, grid_mult: int = 1):
        _check(lib().setb_batch_set_tiling(self.h, int(lz), int(grid_mult)), "setb_batch_set_tiling")

    def tune(self, reps: int = 3):
        lz, gm, ms = C.c_int32(), C.c_int32(), C.c_double()
        _check(lib().setb_batch_tune(self.h, int(reps), C.byref(lz), C.byref(gm), C.byref(ms)), "setb_batch_tune")
        return {"lz": lz.value, "grid_mult": gm.value, "ms_per_stage1": ms.value}
