"""One Cartesian grid split along z: the multi-GPU form of the step.

The reference runs one grid on one GPU (SET_Fortran_Cuda_MHD/cuf_kernel.cuf:780-925).  Here each
rank owns a z slab (setb_init_slab) with two ghost planes on each side; one time step is

    exchange the ghost planes of U  ->  stage 1  ->  (Heun) exchange those of U*  ->  stage 2
    ->  minimum of the next step's dt over all slabs

so the slabs reproduce the single-grid step bit for bit.  The exchange moves 2 planes x 8
variables per neighbour and stage (`exchange_halos`, torch.distributed point-to-point: NCCL over
NVLink between GPUs, gloo on CPU tensors in the tests), the dt minimum is one all-reduce of a
device double.  `LocalSlabs` runs all slabs of a grid on one GPU with device copies for the
exchange: the same slab kernels and ghost-plane protocol, checkable against the single-grid solve
on one device.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import CartDesc, Solver, StepOpts, _check, _dp, _p, lib

GHOST = 2   # ghost planes per side (the reconstruction stencil reaches two planes)


def split_z(nz: int, parts: int) -> list[tuple[int, int]]:
    """(k0, nz_local) of `parts` near-equal slabs of nz planes, each at least GHOST planes."""
    if parts < 1 or nz < GHOST * parts:
        raise ValueError(f"cannot split {nz} planes into {parts} slabs of >= {GHOST} planes")
    base, extra = divmod(nz, parts)
    out, k0 = [], 0
    for r in range(parts):
        n = base + (1 if r < extra else 0)
        out.append((k0, n))
        k0 += n
    return out


class _DeviceArray:
    """__cuda_array_interface__ of a device buffer the library owns (zero-copy torch views)."""

    def __init__(self, ptr: int, shape, strides_elems):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f8", "data": (ptr, False),
                                         "version": 3, "strides": tuple(8 * s for s in strides_elems)}


class SlabSolver(Solver):
    """Planes [k0, k0 + nz_local) of the Cartesian grid `desc`; cell_par holds those planes'
    Cell_par rows ([nx*ny*nz_local, 16], x fastest)."""

    def __init__(self, desc: CartDesc, k0: int, nz_local: int, cell_par: np.ndarray):
        self.desc = desc
        self.k0, self.nz_local = int(k0), int(nz_local)
        self.shape = (self.nz_local, desc.ny, desc.nx)
        self.N = desc.nx * desc.ny * self.nz_local
        cp = np.ascontiguousarray(cell_par, dtype=np.float64)
        assert cp.shape == (self.N, 16)
        h = C.c_void_p()
        _check(lib().setb_init_slab(C.byref(h), C.byref(desc), self.k0, self.nz_local, _p(cp)), "setb_init_slab")
        self.h = h

    def step(self, *a, **k):
        raise RuntimeError("a slab steps stage by stage (SlabRun / LocalSlabs), with its ghost planes exchanged")

    def stage(self, stage: int, opts: StepOpts):
        _check(lib().setb_slab_stage(self.h, int(stage), C.byref(opts)), "setb_slab_stage")

    def view(self, stage: int):
        """(device pointer, var_stride, plane_stride, buffer planes) of the buffer `stage` reads."""
        base, vs, ps, nzb = _dp(), C.c_int64(), C.c_int64(), C.c_int32()
        _check(lib().setb_slab_view(self.h, int(stage), C.byref(base), C.byref(vs), C.byref(ps), C.byref(nzb)),
               "setb_slab_view")
        return C.cast(base, C.c_void_p).value, vs.value, ps.value, nzb.value

    def tensor(self, stage: int):
        """torch view [8, nz_local + 4, plane_stride] of the buffer `stage` reads (no copy)."""
        import torch
        ptr, vs, ps, nzb = self.view(stage)
        return torch.as_tensor(_DeviceArray(ptr, (8, nzb, ps), (vs, ps, 1)), device="cuda")

    def dt_tensor(self):
        """torch view of the device double holding the next step's dt."""
        import torch
        p = _dp()
        _check(lib().setb_slab_dt(self.h, C.byref(p)), "setb_slab_dt")
        return torch.as_tensor(_DeviceArray(C.cast(p, C.c_void_p).value, (1,), (1,)), device="cuda")


def exchange_halos(X, nz_local: int, rank: int, world: int, group=None):
    """Fills the ghost planes of slab buffer X [8, nz_local + 4, plane] from the z neighbours'
    owned edge planes (rank - 1 below, rank + 1 above) with paired point-to-point transfers; the
    ghost planes beyond the grid's z ends are left to setb_slab_stage."""
    import torch
    import torch.distributed as dist
    lo_own, hi_own = X[:, GHOST:2 * GHOST], X[:, nz_local:nz_local + GHOST]
    ops, recv = [], {}
    if rank > 0:
        recv["lo"] = torch.empty_like(lo_own)
        ops += [dist.P2POp(dist.isend, lo_own.contiguous(), rank - 1, group),
                dist.P2POp(dist.irecv, recv["lo"], rank - 1, group)]
    if rank < world - 1:
        recv["hi"] = torch.empty_like(hi_own)
        ops += [dist.P2POp(dist.isend, hi_own.contiguous(), rank + 1, group),
                dist.P2POp(dist.irecv, recv["hi"], rank + 1, group)]
    if ops:
        for r in dist.batch_isend_irecv(ops):
            r.wait()
    if "lo" in recv:
        X[:, 0:GHOST].copy_(recv["lo"])
    if "hi" in recv:
        X[:, nz_local + GHOST:nz_local + 2 * GHOST].copy_(recv["hi"])


def min_dt(dt, group=None):
    """Next step's dt := its minimum over all slabs (in place)."""
    import torch.distributed as dist
    dist.all_reduce(dt, op=dist.ReduceOp.MIN, group=group)


class SlabRun:
    """One rank's slab of a grid decomposed over `world` ranks (torch.distributed initialised).
    Transfers run on the slab's own CUDA stream, so they are ordered with its kernels."""

    def __init__(self, slab: SlabSolver, rank: int, world: int, group=None):
        self.slab, self.rank, self.world, self.group = slab, rank, world, group

    def step(self, nsteps: int, opts: StepOpts):
        import torch
        s = self.slab
        with torch.cuda.stream(torch.cuda.ExternalStream(s.stream())):
            for _ in range(int(nsteps)):
                exchange_halos(s.tensor(1), s.nz_local, self.rank, self.world, self.group)
                s.stage(1, opts)
                if opts.scheme == 2:
                    exchange_halos(s.tensor(2), s.nz_local, self.rank, self.world, self.group)
                    s.stage(2, opts)
                if self.world > 1:
                    min_dt(s.dt_tensor(), self.group)


class LocalSlabs:
    """All z slabs of one grid on this process's GPU: the slab kernels and ghost-plane protocol
    with device copies for the exchange (a check of the decomposition on one device)."""

    def __init__(self, desc: CartDesc, parts: int, cell_par: np.ndarray):
        self.desc = desc
        plane = desc.nx * desc.ny
        cp = np.ascontiguousarray(cell_par, dtype=np.float64)
        self.slabs = [SlabSolver(desc, k0, n, cp[k0 * plane:(k0 + n) * plane]) for k0, n in split_z(desc.nz, parts)]

    def close(self):
        for s in self.slabs:
            s.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _sync(self):
        import torch
        for s in self.slabs:
            _check(s.sync(), "setb_sync")
        torch.cuda.synchronize()

    def _exchange(self, stage: int):
        import torch
        self._sync()
        X = [s.tensor(stage) for s in self.slabs]
        for lo, hi, a, b in zip(self.slabs, self.slabs[1:], X, X[1:]):
            b[:, 0:GHOST].copy_(a[:, lo.nz_local:lo.nz_local + GHOST])
            a[:, lo.nz_local + GHOST:lo.nz_local + 2 * GHOST].copy_(b[:, GHOST:2 * GHOST])
        torch.cuda.synchronize()

    def step(self, nsteps: int, opts: StepOpts):
        import torch
        for _ in range(int(nsteps)):
            self._exchange(1)
            for s in self.slabs:
                s.stage(1, opts)
            if opts.scheme == 2:
                self._exchange(2)
                for s in self.slabs:
                    s.stage(2, opts)
            self._sync()
            dts = [s.dt_tensor() for s in self.slabs]
            m = torch.stack(dts).min()
            for d in dts:
                d.fill_(m.item())
            torch.cuda.synchronize()

    def conserved(self) -> np.ndarray:
        return np.concatenate([s.conserved() for s in self.slabs], axis=1)

    def get_state(self):
        parts = [s.get_state() for s in self.slabs]
        return np.concatenate([p[0] for p in parts]), parts[0][1]
