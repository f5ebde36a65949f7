"""setb_step_noalloc against the handle path (setb_init_cartesian_lism + setb_step).

The no-allocation entry point serves callers that own all device memory themselves and cannot
let the library call cudaMalloc.  Here the test owns the state (a torch tensor, allocated by the
test, never by the entry point), advances it with two calls in a row and checks each result
against the existing entry point on the same problem, with the parity test's per-step bound.
This file is collected last so a failure here comes after every other test has run.
"""
import numpy as np
import pytest

import set_b200 as S
from tests.test_gpu_parity import STEP_TOL, step_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("scheme,order,n_state,calls", [(2, 2, 3, (3, 4)), (1, 1, 2, (3, 2))])
def test_noalloc_matches_handle_path_on_two_calls(scheme, order, n_state, calls):
    import torch
    torch.cuda.set_device(0)
    inflow = S.lism_prim(bmag=0.0 if n_state == 2 else 1.0)
    desc = S.cart_desc((40, 32, 24), inflow=inflow, dt_init=2e-3)
    ic = S.lism_ic(lism=inflow, seed=6)
    o = S.step_opts(n_state=n_state, order=order, scheme=scheme)
    ref = []
    with S.Solver(desc, ic=ic) as s:
        U0 = s.conserved()
        for n in calls:
            t = s.step(n, o)
            ref.append((s.conserved(), t, s.status()))
    N = desc.nx * desc.ny * desc.nz
    U = torch.tensor(U0.reshape(8, N), device="cuda")   # caller-owned, var_stride = N
    stream = torch.cuda.current_stream().cuda_stream
    dt, t = desc.dt_init, 0.0
    floors_before = 0
    for n, (Uref, tref, dref) in zip(calls, ref):
        dt, t, d = S.step_noalloc(desc, o, U.data_ptr(), N, n, dt, t, stream)
        got = U.cpu().numpy().reshape(Uref.shape)
        assert step_err(got, Uref).max() <= STEP_TOL
        assert t == tref and dt == dref.dt_next
        # the handle's counters run since init; the no-alloc call's start at zero each call
        assert d.n_negdens == 0 and d.n_pfloor == dref.n_pfloor - floors_before
        floors_before = dref.n_pfloor


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    desc = S.cart_desc((65, 64, 64))
    U = torch.zeros(8, dtype=torch.float64, device="cuda")
    with pytest.raises(S.SetbError) as e:
        S.step_noalloc(desc, S.step_opts(), U.data_ptr(), 65 * 64 * 64, 1, 1e-3, 0.0)
    assert e.value.code == 9   # SETB_ESIZE
