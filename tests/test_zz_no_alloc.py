"""gdfv_step_noalloc: a predictor-corrector step that allocates no device memory,
for callers that cannot call cudaMalloc (their device memory belongs to their own
pool allocator, or cudaMalloc's latency and implicit synchronisation are not
acceptable in their loop).  Its scratch is a fixed device array inside the library.

The tests call it through the C ABI on device arrays the test owns and check two
calls in a row against the regular stepping entry point (gdfv_run) with the same
dt: per cell to the FP64 parity tolerance of the other GPU tests, and in the float
flux form to their relative-L2 tolerance.  Covered: both flux precisions, both
launch forms (one CTA per tile, and the persistent grid whose tile queue the call
resets), the float corrector's own tile table (56 rows: 7-row tiles), and MHD with
divergence cleaning, whose c_h the call derives from a signal scan of its input,
before any gdfv_run and after one.  This file sorts last so that a run that stops
at the first failure has already run the rest.
"""
import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu

TOL = 1.0e-12
TOL_FP32_L2 = 1.0e-6


def _ptr(t):
    from gdfv._lib import ffi
    return ffi.cast("double*", t.data_ptr())


def _noalloc_steps(sim, U0, dts):
    """Steps of the given dts through gdfv_step_noalloc from U0 (numpy [nq][total])."""
    import torch
    from gdfv._lib import check, ffi
    bad = ffi.new("int*")
    cur = torch.from_numpy(U0.copy()).cuda()
    outs = []
    for dt in dts:
        nxt = torch.empty_like(cur)
        torch.cuda.synchronize()
        check(sim.ctx, sim.L.gdfv_step_noalloc(sim.ctx, _ptr(cur), _ptr(nxt), dt, bad))
        assert bad[0] == 0
        outs.append(nxt.cpu().numpy())
        cur = nxt
    return outs


def _run_steps(sim, n):
    """n regular steps: their dts and the states after each."""
    dts, states = [], []
    for _ in range(n):
        assert sim.run(max_step=1) == 1
        dts.append(sim.time()["dt"])
        states.append(np.concatenate([sim.get_conserved(b) for b in range(len(sim.blocks))], axis=1))
    return dts, states


def _compare(got, ref, fp32, mhd):
    if fp32:
        groups = [(0, 1), (1, 4), (4, 5)] + ([(5, 8)] if mhd else [])
        errs = [cases.rel_l2(got[a:b].ravel(), ref[a:b].ravel()) for a, b in groups]
        assert max(errs) <= TOL_FP32_L2, errs
    else:
        errs = cases.cell_errors(got, ref, mhd)
        assert max(errs.values()) <= TOL, errs


@pytest.mark.parametrize("precision,persistent", [("fp64", False), ("fp64", True), ("fp32", False), ("fp32", True)])
def test_step_noalloc_matches_gdfv_run_twice(precision, persistent):
    import torch
    torch.cuda.init()
    # 56 rows: the float corrector of the no-alloc step (which decodes its stencils from
    # the conserved state) runs over its own 7-row tile table
    case = cases.c2_inflow_box(n=(40, 56, 20), flux="ausmdv", precision=precision)
    sim = cases.build_gpu(case, persistent=persistent)
    assert sim.option("persistent") == int(persistent)
    assert case.nq * sim.total_cells() <= 4194304
    U0 = sim.get_conserved(0)
    dts, refs = _run_steps(sim, 2)
    outs = _noalloc_steps(sim, U0, dts)
    for got, ref in zip(outs, refs):
        _compare(got, ref, precision == "fp32", False)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_step_noalloc_mhd_glm_before_and_after_run(precision):
    """Orszag-Tang with GLM cleaning: c_h comes from the signal of U_in by the step
    controller's rule, so the call matches gdfv_run both before any run (a fresh
    context has no c_h yet) and after a few steps."""
    import torch
    torch.cuda.init()
    case = cases.orszag_tang(n=(64, 64, 4), cleaning=True, precision=precision)
    sim = cases.build_gpu(case)
    U0 = sim.get_conserved(0)
    dts, refs = _run_steps(sim, 2)
    for got, ref in zip(_noalloc_steps(sim, U0, dts), refs):
        _compare(got, ref, precision == "fp32", True)
    assert sim.run(max_step=3) == 3
    U1 = sim.get_conserved(0)
    dts, refs = _run_steps(sim, 2)
    for got, ref in zip(_noalloc_steps(sim, U1, dts), refs):
        _compare(got, ref, precision == "fp32", True)


def test_step_noalloc_rejects_oversize():
    import torch
    from gdfv._lib import GDFV_ERR_ARG, ffi

    case = cases.c2_inflow_box(n=(256, 128, 32), flux="ausmdv")   # 5 * 1,048,576 values > limit
    sim = cases.build_gpu(case)
    u = torch.zeros((5, sim.total_cells()), dtype=torch.float64, device="cuda")
    v = torch.zeros_like(u)
    rc = sim.L.gdfv_step_noalloc(sim.ctx, ffi.cast("double*", u.data_ptr()), ffi.cast("double*", v.data_ptr()),
                                 1e-7, ffi.NULL)
    assert rc == GDFV_ERR_ARG
