"""setb_step_noalloc against the handle path (setb_init_cartesian_lism + setb_step).

The no-allocation entry point serves callers that own all device memory themselves and cannot
let the library call cudaMalloc: a host whose state already lives in its own device arrays, or a
service that reserves HBM up front in its own arena.  Here the test owns the state (a torch
tensor, allocated by the test, never by the entry point), advances it with two calls in a row and
checks each result against the existing entry point on the same problem.

The two paths run the same stage kernels on the same tiles; the handle stages each plane with
tensor copies from its padded device layout, while the caller's layout here is read with plain
loads (odd row pitch and padded variable planes included), so the results are compared bit for
bit as well as with the parity test's per-step bound.
This file is collected last so a failure here comes after every other test has run.
"""
import numpy as np
import pytest

import set_b200 as S
from tests.test_gpu_parity import STEP_TOL, step_err

pytestmark = pytest.mark.gpu


def handle_runs(desc, ic, o, calls):
    out = []
    with S.Solver(desc, ic=ic) as s:
        U0 = s.conserved()
        for n in calls:
            t = s.step(n, o)
            out.append((s.conserved(), t, s.status()))
    return U0, out


def noalloc_runs(desc, o, U0, calls, pad):
    import torch
    N = desc.nx * desc.ny * desc.nz
    vs = N + pad
    U = torch.zeros((8, vs), dtype=torch.float64, device="cuda")   # caller-owned, var_stride = vs
    U[:, :N] = torch.tensor(U0.reshape(8, N), device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    dt, t = desc.dt_init, 0.0
    out = []
    for n in calls:
        dt, t, d = S.step_noalloc(desc, o, U.data_ptr(), vs, n, dt, t, stream)
        out.append((U[:, :N].cpu().numpy().reshape(U0.shape), t, dt, d))
        assert not U[:, N:].any().item()   # the padding of each plane is never written
    return out


@pytest.mark.parametrize("shape,pad", [((40, 32, 24), 0), ((41, 32, 24), 0), ((41, 33, 25), 37)])
@pytest.mark.parametrize("scheme,order,n_state,calls", [(2, 2, 3, (3, 4)), (1, 1, 2, (3, 2))])
def test_noalloc_matches_handle_path_on_two_calls(shape, pad, scheme, order, n_state, calls):
    import torch
    torch.cuda.set_device(0)
    inflow = S.lism_prim(bmag=0.0 if n_state == 2 else 1.0)
    desc = S.cart_desc(shape, inflow=inflow, dt_init=2e-3)
    ic = S.lism_ic(lism=inflow, seed=6)
    o = S.step_opts(n_state=n_state, order=order, scheme=scheme)
    U0, ref = handle_runs(desc, ic, o, calls)
    got = noalloc_runs(desc, o, U0, calls, pad)
    floors_before = 0
    for (Uref, tref, dref), (U, t, dt, d) in zip(ref, got):
        assert step_err(U, Uref).max() <= STEP_TOL
        np.testing.assert_array_equal(U, Uref)   # plain loads and tensor copies: same arithmetic
        assert t == tref and dt == dref.dt_next
        # the handle's counters run since init; the no-alloc call's start at zero each call
        assert d.n_negdens == 0 and d.n_pfloor == dref.n_pfloor - floors_before
        floors_before = dref.n_pfloor


def test_noalloc_second_grid_starts_clean():
    """A call on a different grid after another call leaves nothing behind in the shared
    scratch: its clock, counters and state equal a fresh handle's on that grid."""
    import torch
    torch.cuda.set_device(0)
    o = S.step_opts()
    first = S.cart_desc((48, 40, 36), dt_init=2e-3)
    U0, _ = handle_runs(first, S.lism_ic(seed=2), o, (1,))
    noalloc_runs(first, o, U0, (5,), 0)
    second = S.cart_desc((30, 29, 31), dt_init=1e-3)
    U0b, ref = handle_runs(second, S.lism_ic(seed=9), o, (4,))
    (Uref, tref, dref), = ref
    (U, t, dt, d), = noalloc_runs(second, o, U0b, (4,), 0)
    np.testing.assert_array_equal(U, Uref)
    assert t == tref and dt == dref.dt_next and d.steps == 4 and d.n_pfloor == dref.n_pfloor


def test_noalloc_rejects_sizes_beyond_its_scratch_and_bad_inputs():
    import torch
    U = torch.zeros(8, dtype=torch.float64, device="cuda")
    with pytest.raises(S.SetbError) as e:
        S.step_noalloc(S.cart_desc((65, 64, 64)), S.step_opts(), U.data_ptr(), 65 * 64 * 64, 1, 1e-3, 0.0)
    assert e.value.code == 9   # SETB_ESIZE
    # the handle path's argument checks: bad inflow, bad source, mixed precision
    bad_inflow = S.cart_desc(8, inflow=S.lism_prim(rho=-1.0))
    bad_src = S.cart_desc(8, rho_src=0.0)
    for desc, o in ((bad_inflow, S.step_opts()), (bad_src, S.step_opts()),
                    (S.cart_desc(8), S.step_opts(precision=1))):
        with pytest.raises(S.SetbError) as e:
            S.step_noalloc(desc, o, U.data_ptr(), 512, 1, 1e-3, 0.0)
        assert e.value.code == 1   # SETB_EINVAL
