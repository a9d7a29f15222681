"""gdfv_step_noalloc: a predictor-corrector step that allocates no device memory,
for callers that cannot call cudaMalloc (their device memory belongs to their own
pool allocator, or cudaMalloc's latency and implicit synchronisation are not
acceptable in their loop).  Its scratch is a fixed device array inside the library.

The test calls it through the C ABI on device arrays the test owns and checks
two calls in a row against the regular stepping entry point (gdfv_run) with the
same dt, to the FP64 parity tolerance of the other GPU tests.  This file sorts
last so that a run that stops at the first failure has already run the rest.
"""
import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu

TOL = 1.0e-12


def test_step_noalloc_matches_gdfv_run_twice():
    import torch
    from gdfv._lib import check, ffi

    torch.cuda.init()
    case = cases.c2_inflow_box(n=(40, 24, 20), flux="ausmdv")
    sim = cases.build_gpu(case)
    L, h = sim.L, sim.ctx
    nq, n = case.nq, sim.total_cells()
    assert nq * n <= 4194304

    U0 = sim.get_conserved(0)
    u_in = torch.from_numpy(U0.copy()).cuda()
    u_out = torch.empty_like(u_in)
    u_out2 = torch.empty_like(u_in)
    torch.cuda.synchronize()

    # reference: one regular step, its dt, and the state it produced
    assert sim.run(max_step=1) == 1
    dt1 = sim.time()["dt"]
    ref1 = sim.get_conserved(0)
    assert sim.run(max_step=1) == 1
    dt2 = sim.time()["dt"]
    ref2 = sim.get_conserved(0)

    bad = ffi.new("int*")
    p = lambda t: ffi.cast("double*", t.data_ptr())
    check(h, L.gdfv_step_noalloc(h, p(u_in), p(u_out), dt1, bad))
    assert bad[0] == 0
    out1 = u_out.cpu().numpy()
    check(h, L.gdfv_step_noalloc(h, p(u_out), p(u_out2), dt2, bad))
    assert bad[0] == 0
    out2 = u_out2.cpu().numpy()

    for got, ref in ((out1, ref1), (out2, ref2)):
        errs = cases.cell_errors(got, ref, False)
        assert max(errs.values()) <= TOL, errs


def test_step_noalloc_rejects_oversize():
    from gdfv._lib import GDFV_ERR_ARG, ffi

    case = cases.c2_inflow_box(n=(256, 128, 32), flux="ausmdv")   # 5 * 1,048,576 values > limit
    sim = cases.build_gpu(case)
    import torch
    u = torch.zeros((5, sim.total_cells()), dtype=torch.float64, device="cuda")
    v = torch.zeros_like(u)
    rc = sim.L.gdfv_step_noalloc(sim.ctx, ffi.cast("double*", u.data_ptr()), ffi.cast("double*", v.data_ptr()),
                                 1e-7, ffi.NULL)
    assert rc == GDFV_ERR_ARG
