"""torch.autograd wrappers over the hand-written adjoint kernels.

* `residual(sim, U)`: R(U) with backward = gdfv_residual_vjp.
* `jvp(sim, U, v)`: J v by the real Frechet derivative (gdfv_residual_jvp), the
  Jacobian-vector product of a Newton-Krylov solver.
* `rollout(sim, U0, theta, nsteps, checkpoint_every=None)`: nsteps predictor-corrector
  steps of the GPU solver from U0, differentiable in U0 and in the supersonic-
  inflow state theta = (p, T, vel.x), which the forward sets on every supersonic-
  inflow face (the other components of each face's state stay as configured), so
  that dJ/dtheta sums the cotangents of all those faces.  The forward records each step's dt and
  keeps a copy of the state every `checkpoint_every` steps (None: the whole
  trajectory stays resident in device memory when it fits, see resident_steps, and
  the backward recomputes nothing); the backward
  (gdfv_rollout_adjoint) recomputes each segment from its checkpoint
  (bit-identical to the forward steps) on a second stream while it applies the
  adjoint of the predictor-corrector step (e4/simcore_gasdynamic_step.d:1245-1333)
  to the segment after it; the last segment's states and predictor states are
  kept by the forward as it takes the steps, so that segment is not recomputed:
      U1 = U0 + dt R(U0),  U2 = U0 + dt (R(U0)/2 + R(U1)/2)
      mu  = J(U1)^T (dt/2 lam)
      lam <- lam + mu + J(U0)^T (dt/2 lam + dt mu)
  with dt frozen at its forward value (the CFL rule is not differentiated).  MHD
  rollouts with GLM cleaning hold each step's c_h fixed likewise, and the step's psi
  damping D enters as U1 -> D U1 in the corrector and U2 -> D U2.
Tensors are float64 on the simulation's device, shaped [nq, total cells].
"""
import torch

from ._lib import GDFV_ERR_STATE, GDFV_OK, check, ffi


def _p(t):
    return ffi.cast("double*", t.data_ptr())


def vjp(sim, U, W):
    """G = (dR/dU)^T W and the inflow-state cotangents [n_inflow, 6] (rho, vel, u, a; MHD
    [n_inflow, 10]: and B, psi)."""
    U = U.contiguous()
    W = W.contiguous()
    G = torch.empty_like(U)
    n_in = max(1, getattr(sim, "n_inflow", 1))
    gin = torch.zeros((n_in, 10 if sim.nq == 10 else 6), dtype=torch.float64)
    torch.cuda.current_stream().synchronize()
    check(sim.ctx, sim.L.gdfv_residual_vjp(sim.ctx, _p(U), _p(W), _p(G), ffi.cast("double*", gin.data_ptr())))
    return G, gin


def jvp(sim, U, v, R0=None, sigma=0.0):
    """Jv by the real Frechet derivative as evalJacobianVecProd computes it
    (gdfv_residual_jvp); sigma <= 0 takes the Knoll-McHugh perturbation.
    Returns (Jv, sigma used)."""
    U = U.contiguous()
    v = v.contiguous()
    Jv = torch.empty_like(U)
    used = ffi.new("double*")
    torch.cuda.current_stream().synchronize()
    check(sim.ctx, sim.L.gdfv_residual_jvp(sim.ctx, _p(U), _p(v), _p(R0.contiguous()) if R0 is not None else ffi.NULL,
                                           float(sigma), _p(Jv), used))
    return Jv, used[0]


def residual_eval(sim, U):
    U = U.contiguous()
    R = torch.empty_like(U)
    torch.cuda.current_stream().synchronize()
    sim.residual(U.data_ptr(), R.data_ptr())
    return R


def step_dt(sim, U, dt, with_predictor=False):
    """One step of the given dt; with_predictor also returns U1 = U + dt R(U)."""
    U = U.contiguous()
    out = torch.empty_like(U)
    U1 = torch.empty_like(U) if with_predictor else None
    torch.cuda.current_stream().synchronize()
    check(sim.ctx, sim.L.gdfv_step_dt(sim.ctx, _p(U), _p(out), float(dt), _p(U1) if with_predictor else ffi.NULL))
    return (out, U1) if with_predictor else out


def steps_dt(sim, U, dts, outs, preds):
    """Chain of fixed-dt steps from U: outs[m] after step m, preds[m] its predictor
    state (one host synchronisation at the end)."""
    n = len(dts)
    po = ffi.new("double*[]", [_p(t) for t in outs[:n]])
    pp = ffi.new("double*[]", [_p(t) for t in preds[:n]])
    pd = ffi.new("double[]", [float(d) for d in dts])
    torch.cuda.current_stream().synchronize()
    check(sim.ctx, sim.L.gdfv_steps_dt(sim.ctx, _p(U.contiguous()), po, pp, pd, n))


def step_adjoint(sim, U0, U1, dt, lam, gin):
    """lam <- (dU2/dU0)^T lam for the predictor-corrector step U0 -> U2 of frozen dt
    (U1 its predictor state), in place; inflow cotangents added into gin [n_inflow, 6]
    (MHD: [n_inflow, 10]) on the device.  Enqueued without a host synchronisation."""
    check(sim.ctx, sim.L.gdfv_step_adjoint(sim.ctx, _p(U0), _p(U1), float(dt), _p(lam), _p(gin)))


class Residual(torch.autograd.Function):
    @staticmethod
    def forward(ctx, U, sim):
        ctx.sim = sim
        ctx.save_for_backward(U)
        return residual_eval(sim, U)

    @staticmethod
    def backward(ctx, gR):
        (U,) = ctx.saved_tensors
        G, _ = vjp(ctx.sim, U, gR)
        return G, None


def residual(sim, U):
    return Residual.apply(U, sim)


def inflow_chain(sim, theta, gprim):
    """d/d(p, T, vel.x) of an inflow ghost state (FlowState:new{p=,T=}: rho = p/(R T),
    u = Cv T, a = sqrt(gamma R T)) from its cotangent (rho, vx, vy, vz, u, a; an MHD
    state's B and psi cotangents follow and do not enter)."""
    p, T, _ = [float(x) for x in theta]
    R, g = sim.gas.R, sim.gas.gamma
    Cv = R / (g - 1.0)
    a = (g * R * T) ** 0.5
    gr, gvx, _, _, gu, ga = [float(x) for x in gprim[:6]]
    dp = gr / (R * T)
    dT = gr * (-p / (R * T * T)) + gu * Cv + ga * g * R / (2.0 * a)
    return torch.tensor([dp, dT, gvx], dtype=torch.float64)


class Rollout(torch.autograd.Function):
    @staticmethod
    def forward(ctx, U0, theta, sim, nsteps, checkpoint_every):
        U0 = U0.contiguous()
        K = min(checkpoint_every, nsteps)
        dts, ckpts = [], {0: U0.clone()}
        # work arrays of the backward (two sets of K states and K predictor states);
        # the first set keeps the last segment's steps as the forward takes them.  One
        # segment (K = nsteps) needs only that set: the backward reads no other.
        work = [torch.empty_like(U0) for _ in range((2 if K == nsteps else 4) * K)]
        outs0, preds0 = work[:K], work[K:2 * K]
        s_last = ((nsteps + K - 1) // K - 1) * K
        # theta is the state of every supersonic-inflow face for this rollout
        p, T, vx = [float(x) for x in theta.detach().cpu()]
        for i, st in enumerate(sim.inflow_states()):
            s = st.copy()
            s[0], s[1], s[2] = p, T, vx
            sim.set_inflow(i, s)
        # what each step leaves: a checkpoint, or (last segment) its state and predictor state
        states, preds = [None] * nsteps, [None] * nsteps
        for n in range(nsteps):
            if (n + 1) % K == 0 and n + 1 < nsteps:
                ckpts[n + 1] = torch.empty_like(U0)
                states[n] = ckpts[n + 1]
            if n >= s_last:
                preds[n] = preds0[n - s_last]
                if n < nsteps - 1:
                    states[n] = outs0[n - s_last]
        ptr = lambda t: ffi.NULL if t is None else _p(t)
        pst = ffi.new("double*[]", [ptr(t) for t in states])
        ppr = ffi.new("double*[]", [ptr(t) for t in preds])
        hdt = ffi.new("double[]", nsteps)
        recorded = False
        for attempt in range(2):
            sim.set_time(0.0, 0, sim.config.dt_init)
            torch.cuda.current_stream().synchronize()
            state = _state_view(sim)
            state.copy_(U0)
            torch.cuda.synchronize()
            if attempt == 0:
                # all steps and their records on the device, one host round trip
                rc = sim.L.gdfv_run_record(sim.ctx, nsteps, pst, ppr, hdt)
                if rc == GDFV_OK:
                    dts = [hdt[n] for n in range(nsteps)]
                    recorded = True
                    break
                if rc != GDFV_ERR_STATE:
                    check(sim.ctx, rc)
                # a step was retried: take the steps one by one below
        if not recorded:
            for n in range(nsteps):
                sim.run(max_step=1)
                dts.append(sim.time()["dt"])
                if n >= s_last:
                    m = n - s_last
                    U0n = ckpts[s_last] if m == 0 else outs0[m - 1]
                    check(sim.ctx, sim.L.gdfv_last_predictor_state(sim.ctx, _p(U0n), _p(preds0[m])))
                if states[n] is not None:
                    states[n].copy_(_state_view(sim))
                    torch.cuda.synchronize()
        UN = _state_view(sim).clone()
        torch.cuda.synchronize()
        sim.rollout_recorded = recorded   # False: a retried step sent the forward step by step
        ctx.sim, ctx.dts, ctx.ckpts, ctx.k, ctx.work = sim, dts, ckpts, K, work
        ctx.theta = theta.detach().clone()
        return UN

    @staticmethod
    def backward(ctx, gUN):
        sim, dts, ckpts, K = ctx.sim, ctx.dts, ctx.ckpts, ctx.k
        lam = gUN.contiguous().clone()
        # the inflow ghost state's cotangents: rho, vel, u, a (MHD: and B, psi)
        gin = torch.zeros((max(1, getattr(sim, "n_inflow", 1)), 10 if sim.nq == 10 else 6), dtype=torch.float64,
                          device=lam.device)
        nseg = (len(dts) + K - 1) // K
        pc = ffi.new("double*[]", [_p(ckpts[s * K]) for s in range(nseg)])
        sets = ctx.work if len(ctx.work) == 4 * K else ctx.work + ctx.work
        pw = ffi.new("double*[]", [_p(t) for t in sets])
        pd = ffi.new("double[]", [float(d) for d in dts])
        torch.cuda.synchronize()
        check(sim.ctx, sim.L.gdfv_rollout_adjoint(sim.ctx, pc, nseg, pd, len(dts), K, pw, 1, _p(lam), _p(gin)))
        ctx.work = None
        gin = gin.cpu()
        gtheta = sum(inflow_chain(sim, ctx.theta, gin[i]) for i in range(max(1, sim.n_inflow)))
        gtheta = gtheta.to(ctx.theta.device)
        return lam, gtheta, None, None, None


def _state_view(sim):
    """The library's current state buffer as a torch tensor (no copy)."""
    return _from_ptr(sim.state_ptr(), (sim.nq, sim.total_cells()))


def _from_ptr(ptr, shape):
    import numpy as np
    numel = int(np.prod(shape))

    class _Holder:
        __cuda_array_interface__ = {"shape": (numel,), "typestr": "<f8", "data": (ptr, False), "version": 3}

    return torch.as_tensor(_Holder(), device="cuda").view(*shape)


def resident_steps(sim, nsteps, fraction=0.5):
    """The checkpoint interval that keeps a whole rollout of nsteps resident (nsteps), when
    its states and predictor states fit in `fraction` of the free device memory and
    nsteps <= 64 (8.4 GB for 50 steps of 1M Euler cells); else 10."""
    state_bytes = 8 * sim.nq * sim.total_cells()
    free, _ = torch.cuda.mem_get_info()
    if nsteps <= 64 and 2 * nsteps * state_bytes <= fraction * free:
        return int(nsteps)
    return 10


def rollout(sim, U0, theta, nsteps, checkpoint_every=None):
    K = resident_steps(sim, nsteps) if checkpoint_every is None else int(checkpoint_every)
    return Rollout.apply(U0, theta, sim, int(nsteps), K)
