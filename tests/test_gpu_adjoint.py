"""GPU adjoint: the hand-written VJP of R(U) (gdfv_residual_vjp) and the
checkpointed rollout adjoint behind torch.autograd.Function.

Checks, all in FP64 (ausmdv, and hllc where named):
* <w, J v> from the oracle's complex-step JVP (e4/steadystate_core.d:1972-2060
  restated, src/ntypes/complex.d semantics) equals <J^T w, v> from the VJP kernel;
* the same against the oracle's real Frechet JVP with the Knoll-McHugh step
  (e4/steadystate_core.d:1878-1970, :3040-3078), to its truncation error;
* dJ/dU0 and dJ/d(inflow p, T, u) through a multi-step rollout with checkpoints
  against central finite differences (relative step 1e-6), J the pressure
  integral over the y-min wall.
"""
import numpy as np
import pytest
import torch

import cases

pytestmark = pytest.mark.gpu


def _gpu_to_oracle_layout(case, X):
    """[nq][total] (blocks concatenated per variable) -> the oracle's block-major SoA."""
    out, off = [], 0
    for b in case.blocks:
        n = int(np.prod(b["n"]))
        out.append(X[:, off:off + n].ravel())
        off += n
    return np.concatenate(out)


def _state_after(case, nsteps):
    orc, sim = cases.build_pair(case)
    assert sim.run(max_step=nsteps) == nsteps
    if case.mhd:   # the oracle takes the same steps, so that both hold the same c_h
        assert orc.run(nsteps) == 0
    U = np.concatenate([sim.get_conserved(b) for b in range(len(case.blocks))], axis=1)
    for b in range(len(case.blocks)):   # the oracle evaluates at the same state
        assert orc.set_U(b, sim.get_conserved(b)) == 0
    return orc, sim, U


def _dot_check(case, steps, tol, frechet=False, seed=0):
    from gdfv.autograd import vjp
    orc, sim, U = _state_after(case, steps)
    rng = np.random.default_rng(seed)
    scale = np.abs(U).max(axis=1, keepdims=True)
    v = rng.standard_normal(U.shape) * scale
    w = rng.standard_normal(U.shape)
    Uo, vo = _gpu_to_oracle_layout(case, U), _gpu_to_oracle_layout(case, v)
    if frechet:
        Jv, _ = orc.jvp_real(Uo, vo)
    else:
        Jv = orc.jvp_complex(Uo, vo)
    lhs = float(np.dot(_gpu_to_oracle_layout(case, w), Jv))
    G, _ = vjp(sim, torch.from_numpy(U).cuda(), torch.from_numpy(w).cuda())
    rhs = float(np.sum(G.cpu().numpy() * v))
    assert abs(lhs - rhs) <= tol * max(abs(lhs), abs(rhs)), (lhs, rhs)


def test_vjp_transpose_of_complex_step_jvp():
    _dot_check(cases.c2_inflow_box(n=(24, 16, 12)), 6, 1e-10)


def test_vjp_transpose_of_complex_step_jvp_shock_box():
    _dot_check(cases.c1_shock_box(n=16), 8, 1e-10, seed=1)


def test_vjp_transpose_multiblock_exchange():
    _dot_check(cases.multiblock_lattice(nb=(2, 1, 2), sizes=(16, 24), seed=3), 4, 1e-10, seed=2)


def test_vjp_transpose_hllc():
    """hllc (e4/fluxcalc.d:653-820): the reverse of its Roe-averaged wave speeds, the
    star state and the side and star switches; the supersonic inflow box (mostly the
    upwind side alone) and the subsonic shock box (star states on both sides)."""
    _dot_check(cases.c2_inflow_box(n=(24, 16, 12), flux="hllc", noise_all=True), 6, 1e-10, seed=8)
    box = cases.c1_shock_box(n=16)
    box.config["flux_calculator"] = "hllc"
    _dot_check(box, 8, 1e-10, seed=9)


@pytest.mark.parametrize("flux", ["ausmdv", "hllc"])
def test_vjp_transpose_2d(flux):
    """2D blocks: four faces per cell (no k faces), areas and volumes per unit depth."""
    case = cases.c2_inflow_box(n=(40, 24, 1), flux=flux, noise_all=True)
    case.config["dimensions"] = 2
    _dot_check(case, 6, 1e-10, seed=10)


@pytest.mark.parametrize("flux", ["ausmdv", "hllc"])
def test_vjp_transpose_graded_blocks(flux):
    """Graded (stretched rectilinear) blocks: each side of a face reconstructs with its own
    cell's l2r2 weights, the face's area comes from its cells' lengths and each side
    divides by its own volume; the lattice joins four differently graded blocks by
    exchange."""
    _dot_check(cases.graded_inflow_box(flux=flux), 6, 1e-10, seed=13)
    if flux == "ausmdv":
        _dot_check(cases.graded_lattice(), 6, 1e-10, seed=14)


@pytest.mark.parametrize("case_name", ["orszag_tang", "orszag_tang_no_cleaning", "slip_dipole", "shock_tube_2d"])
def test_vjp_transpose_mhd(case_name):
    """The MHD residual (hlle with GLM, e4/fluxcalc.d:54-187, :1608-1780): the reverse of
    the fast magnetosonic speeds, the one-sided fluxes and jumps, the GLM terms of F[B]
    and F[psi] and F[divB], the MHD decode; periodic exchange (Orszag-Tang, with and
    without divergence cleaning), slip walls whose ghosts carry the dipole field, and the
    2D MHD shock tube (extrapolation and exchange; its states jittered, since the plain
    tube's uniform regions meet the disturbed ones one ulp apart, where the clipping
    switches follow each side's own rounding).  c_h is the context's, frozen."""
    case = {"orszag_tang": lambda: cases.orszag_tang(n=(24, 24, 4)),
            "orszag_tang_no_cleaning": lambda: cases.orszag_tang(n=(24, 24, 4), cleaning=False),
            "slip_dipole": lambda: cases.mhd_slip_dipole(n=(24, 20, 4)),
            "shock_tube_2d": lambda: cases.mhd_shock_tube(N=64, noise=0.01)}[case_name]()
    _dot_check(case, 4, 1e-10, seed=16)


def test_vjp_transpose_lmr_limiter():
    """van_albada_variant lmr (lmr/onedinterp.d:147-151): each face's epsilon scales with
    the larger of its two states, which adds a derivative through epsilon (taken at 1e-3
    so that it weighs)."""
    for case in (cases.c1_shock_box(n=16), cases.c2_inflow_box(n=(24, 16, 12), noise_all=True)):
        case.config.update(van_albada_variant="lmr", epsilon_van_albada=1e-3)
        _dot_check(case, 6, 1e-10, seed=12)


@pytest.mark.parametrize("bc", ["simple_flux", "fixed_p", "fixed_pt"])
def test_vjp_transpose_outflow_boundaries(bc):
    """OutFlowBC_SimpleFlux (the boundary face's flux from the interior cell alone, on
    faces the flow leaves and on closed ones), OutFlowBC_FixedP and OutFlowBC_FixedPT
    (ghost rho and u from the outside p, or p and T) on the subsonic shock box, whose flow
    runs both ways through its x faces."""
    from test_gpu_parity import OUTFLOW_BCS, _with_bcs
    _dot_check(_with_bcs(cases.c1_shock_box(n=16), OUTFLOW_BCS[bc]), 8, 1e-10, seed=11)


def test_vjp_transpose_oriented_and_rotating_exchanges():
    """Exchange ghosts placed by orientation 3 (the cotangent goes to the partner cell
    the map names), and ghosts whose velocity the exchange turns by +-90 degrees
    (the cotangent goes back through the transpose of the rotation)."""
    _dot_check(cases.exchange_pair(3), 4, 1e-10, seed=5)
    _dot_check(cases.quarter_rotational(n=(16, 16, 4), seed=7), 4, 1e-10, seed=6)


def test_vjp_against_reference_frechet_jvp():
    _dot_check(cases.c2_inflow_box(n=(24, 16, 12)), 6, 1e-5, frechet=True, seed=4)


def wall_pressure(case, U, R):
    """J = sum over y-min wall faces of p_face * area; at a slip wall with extrema
    clipping the reconstructed face pressure equals the wall cell's pressure."""
    nic, njc, nkc = case.blocks[0]["n"]
    dx, dy, dz = case.blocks[0]["d"]
    g = case.gamma
    Cvinv = (g - 1.0) / R
    Uv = U.view(U.shape[0], nkc, njc, nic)[:, :, 0, :]
    rho = Uv[0]
    dinv = 1.0 / rho
    v0, v1, v2 = Uv[1] * dinv, Uv[2] * dinv, Uv[3] * dinv
    u = Uv[4] * dinv - 0.5 * (v0 * v0 + v1 * v1 + v2 * v2)
    p = rho * R * (u * Cvinv)
    return (p * (dx * dz)).sum()


def _rollout_fd_check(extra_config, steps_tols, p_tols):
    """Gradient of J through a 12-step checkpointed rollout (checkpoint every 5 steps)
    against central differences along two random directions in U0 and along the
    inflow pressure, replaying the forward's dt sequence."""
    from gdfv.autograd import rollout, step_dt
    case = cases.c2_inflow_box(n=(24, 16, 12), noise_all=True)
    case.config.update(extra_config)
    inf = cases.inflow_state_m3()
    _, sim = cases.build_pair(case)
    U0 = torch.from_numpy(sim.get_conserved(0)).cuda()
    theta = torch.tensor([inf["p"], inf["T"], inf["vel"][0]], dtype=torch.float64, requires_grad=True)
    U0r = U0.clone().requires_grad_(True)
    nsteps, K = 12, 5
    UN = rollout(sim, U0r, theta, nsteps, K)
    J = wall_pressure(case, UN, case.R)
    J.backward()
    gU0 = U0r.grad.detach()
    _, sim_r = cases.build_pair(case)
    dts = []
    for _ in range(nsteps):
        sim_r.run(max_step=1)
        dts.append(sim_r.time()["dt"])

    def J_of(U, s):
        X = U
        for dt in dts:
            X = step_dt(s, X, dt)
        return float(wall_pressure(case, X, case.R))

    rng = np.random.default_rng(7)
    scale = torch.from_numpy(np.abs(U0.cpu().numpy()).max(axis=1, keepdims=True)).cuda()
    vs = [torch.from_numpy(rng.standard_normal(tuple(U0.shape))).cuda() * scale for _ in range(2)]
    ads = [float((gU0 * v).sum()) for v in vs]
    floor = 0.1 * max(abs(a) for a in ads)   # a direction nearly orthogonal to the gradient
    for trial, (v, ad) in enumerate(zip(vs, ads)):
        for h, tol in steps_tols:
            fd = (J_of(U0 + h * v, sim_r) - J_of(U0 - h * v, sim_r)) / (2 * h)
            assert abs(fd - ad) <= tol * max(abs(fd), abs(ad), floor), (trial, h, fd, ad)
    for rel, tol in p_tols:
        hp = rel * inf["p"]
        vals = []
        for sgn in (1, -1):
            c2 = cases.c2_inflow_box(n=(24, 16, 12), noise_all=True)
            c2.config.update(extra_config)
            c2.blocks[0]["bcs"]["west"][1]["inflow"] = dict(inf, p=inf["p"] + sgn * hp)
            vals.append(J_of(U0, cases.build_gpu(c2)))
        fd_p = (vals[0] - vals[1]) / (2 * hp)
        assert abs(fd_p - float(theta.grad[0])) <= tol * abs(fd_p), (rel, fd_p, float(theta.grad[0]))


def test_rollout_gradients_against_finite_differences():
    """Default options (van Albada limiter, extrema clipping).  A central difference
    straddles limiter corners (del*dLm = 0) in a fraction of faces proportional to
    its step, so it converges to the derivative only linearly: observed up to 6e-3
    at the relative step 1e-6 and 1e-5 at 1e-8 over 12 steps (worst on directions
    with a small derivative).  Asserted with margins above those; the strict check
    is the smooth configuration below."""
    _rollout_fd_check({}, ((1e-6, 2e-2), (1e-8, 1e-3)), ((1e-6, 2e-2), (1e-8, 1e-3)))


def test_rollout_gradients_hllc_smooth_configuration():
    """The same with hllc: the checkpointed rollout adjoint through the hllc VJP."""
    _rollout_fd_check(dict(flux_calculator="hllc", apply_limiter=False, extrema_clipping=False),
                      ((1e-6, 1e-4), (1e-7, 2e-5)), ((1e-6, 1e-4), (1e-7, 2e-5)))


def test_rollout_gradients_smooth_configuration():
    """Limiter and clipping off: central differences converge quadratically down to
    the relative step 1e-6; at 1e-7 the error (observed 2e-7 on a direction whose
    derivative is 3e-4) is roundoff in J, not truncation."""
    _rollout_fd_check(dict(apply_limiter=False, extrema_clipping=False), ((1e-6, 1e-4), (1e-7, 2e-5)),
                      ((1e-6, 1e-4), (1e-7, 2e-5)))


@pytest.mark.parametrize("checkpoint_every", [5, None])
def test_rollout_gradients_mhd_without_cleaning(checkpoint_every):
    """MHD rollouts (hlle, no divergence cleaning): the step adjoint's chain through the
    MHD decode, face and reverse-decode kernels, checkpointed (every 5 of 12 steps) and
    resident.  Orszag-Tang 24x24x4 in the smooth configuration (limiter and clipping
    off, so that central differences converge quadratically); J = <W, U_N> with fixed
    random weights; the forward's dt sequence replayed for the differences."""
    from gdfv.autograd import rollout, step_dt
    case = cases.orszag_tang(n=(24, 24, 4), cleaning=False)
    case.config.update(apply_limiter=False, extrema_clipping=False)
    _, sim = cases.build_pair(case)
    U0 = torch.from_numpy(sim.get_conserved(0)).cuda()
    rng = np.random.default_rng(11)
    W = torch.from_numpy(rng.standard_normal(tuple(U0.shape))).cuda()
    theta = torch.tensor([1.0, 1.0, 0.0], dtype=torch.float64, requires_grad=True)   # no inflow faces
    U0r = U0.clone().requires_grad_(True)
    nsteps = 12
    UN = rollout(sim, U0r, theta, nsteps, checkpoint_every)
    (UN * W).sum().backward()
    gU0 = U0r.grad.detach()
    assert float(theta.grad.abs().sum()) == 0.0
    _, sim_r = cases.build_pair(case)
    dts = []
    for _ in range(nsteps):
        sim_r.run(max_step=1)
        dts.append(sim_r.time()["dt"])

    def J_of(U):
        X = U
        for dt in dts:
            X = step_dt(sim_r, X, dt)
        return float((X * W).sum())

    assert abs(J_of(U0) - float((UN.detach() * W).sum())) <= 1e-12 * abs(J_of(U0))
    scale = torch.from_numpy(np.abs(U0.cpu().numpy()).max(axis=1, keepdims=True)).cuda()
    scale[9] = 1.0   # divB starts at 0
    for trial in range(2):
        v = torch.from_numpy(rng.standard_normal(tuple(U0.shape))).cuda() * scale
        ad = float((gU0 * v).sum())
        h = 1e-6
        fd = (J_of(U0 + h * v) - J_of(U0 - h * v)) / (2 * h)
        assert abs(fd - ad) <= 1e-5 * max(abs(fd), abs(ad)), (trial, fd, ad)


def test_fixed_dt_steps_mhd_cleaning_replay_gdfv_run():
    """With GLM cleaning each step's c_h follows the signal of its start state: the
    fixed-dt steps (gdfv_step_dt, and the chains gdfv_steps_dt that recompute a rollout's
    segments) form it as gdfv_run does -- a scan of the chain's input, then the maxima
    each corrector leaves -- and replay gdfv_run's steps bit for bit."""
    from gdfv.autograd import step_dt, steps_dt
    case = cases.orszag_tang(n=(24, 24, 4))
    _, sim = cases.build_pair(case)
    U0 = torch.from_numpy(sim.get_conserved(0)).cuda()
    states, dts = [], []
    for _ in range(5):
        sim.run(max_step=1)
        dts.append(sim.time()["dt"])
        states.append(sim.get_conserved(0))
    _, sim_r = cases.build_pair(case)
    X = U0
    for n, dt in enumerate(dts):
        X = step_dt(sim_r, X, dt)
        assert np.array_equal(X.cpu().numpy(), states[n]), n
    outs = [torch.empty_like(U0) for _ in dts]
    preds = [torch.empty_like(U0) for _ in dts]
    steps_dt(sim_r, U0, dts, outs, preds)
    for n in range(len(dts)):
        assert np.array_equal(outs[n].cpu().numpy(), states[n]), n


def test_step_adjoint_mhd_with_cleaning_against_oracle():
    """The step adjoint with GLM cleaning is the transpose of the step's Jacobian at
    frozen dt and c_h: U2 = D (U0 + dt/2 R(U0) + dt/2 R(D U1)), U1 = U0 + dt R(U0), D
    damping psi by exp(-c_h dt / (0.18 L)) (e4/fvcell.d:1068-1074).  J_step v is
    composed from the oracle's complex-step residual JVPs at U0 and D U1 with the GPU
    step's c_h; <lam, J_step v> = <J_step^T lam, v> to 1e-10."""
    from gdfv.autograd import step_adjoint
    from gdfv._lib import ffi
    case = cases.orszag_tang(n=(24, 24, 4))
    orc, sim = cases.build_pair(case)
    sim.run(max_step=3)   # psi away from zero
    U0 = torch.from_numpy(sim.get_conserved(0)).cuda()
    sim.run(max_step=1)
    t = sim.time()
    dt, c_h = t["dt"], t["c_h"]
    U1 = torch.empty_like(U0)
    assert sim.L.gdfv_last_predictor_state(sim.ctx, ffi.cast("double*", U0.data_ptr()),
                                           ffi.cast("double*", U1.data_ptr())) == 0
    torch.cuda.synchronize()
    damp = np.exp(-(c_h * c_h / (0.18 * 1.0 * c_h)) * dt)
    assert 0.0 < damp < 1.0
    D = np.ones((10, 1))
    D[8] = damp
    rng = np.random.default_rng(21)
    U0n, U1n = U0.cpu().numpy(), U1.cpu().numpy()
    v = rng.standard_normal(U0n.shape) * np.maximum(np.abs(U0n).max(axis=1, keepdims=True), 1e-3)
    lam = rng.standard_normal(U0n.shape)
    orc.set("c_h", c_h)   # the residual JVPs take the step's c_h
    lay = lambda X: _gpu_to_oracle_layout(case, X)
    unlay = lambda x: x.reshape(U0n.shape)   # one block: the same [nq][cells] order
    J0v = unlay(orc.jvp_complex(lay(U0n), lay(v)))
    w1 = D * (v + dt * J0v)
    J1w = unlay(orc.jvp_complex(lay(D * U1n), lay(w1)))
    JSv = D * (v + 0.5 * dt * J0v + 0.5 * dt * J1w)
    lhs = float(np.sum(lam * JSv))
    lam_t = torch.from_numpy(lam.copy()).cuda()
    gin = torch.zeros((1, 10), dtype=torch.float64, device="cuda")
    step_adjoint(sim, U0, U1, dt, lam_t, gin)
    torch.cuda.synchronize()
    rhs = float(np.sum(lam_t.cpu().numpy() * v))
    assert abs(lhs - rhs) <= 1e-10 * max(abs(lhs), abs(rhs)), (lhs, rhs)


def test_mhd_rollout_with_cleaning_resident_matches_checkpointed():
    """MHD rollout with GLM cleaning: the checkpointed backward recomputes each segment
    with each step's c_h and damps psi as the forward did, so its gradients equal the
    resident trajectory's to the rounding of the FP64 atomic accumulation."""
    from gdfv.autograd import rollout
    case = cases.orszag_tang(n=(24, 24, 4))
    _, sim = cases.build_pair(case)
    U0 = torch.from_numpy(sim.get_conserved(0)).cuda()
    W = torch.from_numpy(np.random.default_rng(4).standard_normal(tuple(U0.shape))).cuda()
    grads = []
    for K in (9, 3):
        theta = torch.tensor([1.0, 1.0, 0.0], dtype=torch.float64, requires_grad=True)
        U0r = U0.clone().requires_grad_(True)
        UN = rollout(sim, U0r, theta, 9, K)
        (UN * W).sum().backward()
        grads.append(U0r.grad.clone())
    assert float(grads[0][8].abs().max()) > 0.0   # psi carries a cotangent
    assert torch.allclose(grads[0], grads[1], rtol=1e-11, atol=1e-11 * float(grads[1].abs().max()))


def test_rollout_theta_drives_every_inflow_face():
    """The rollout's inflow state theta = (p, T, vel.x) is the state of every
    supersonic-inflow face in the forward: at a theta other than the configured one,
    on a lattice with two inflow faces, the rollout's final state equals (bit for bit)
    a run of a simulation configured with theta, and dJ/dtheta -- the cotangents of
    both faces summed -- matches central differences in p and T (limiter and clipping
    off, so the differences converge quadratically)."""
    from gdfv.autograd import rollout, step_dt
    smooth = dict(apply_limiter=False, extrema_clipping=False)
    inf = cases.inflow_state_m3()

    def make(inflow):
        c = cases.multiblock_lattice(nb=(1, 2, 1), sizes=(16,), seed=3)
        c.config.update(smooth)
        for b in c.blocks:
            if b["bcs"]["west"][0] == "inflow_supersonic":
                b["bcs"]["west"] = ("inflow_supersonic", dict(inflow=inflow))
        return c

    def state(s):
        return np.concatenate([s.get_conserved(b) for b in range(2)], axis=1)

    def load(s, U):
        n = U.shape[1] // 2
        for b in range(2):
            s.set_conserved(b, U[:, b * n:(b + 1) * n])

    inf2 = dict(inf, p=inf["p"] * 1.05, T=inf["T"] * 0.98)
    _, sim = cases.build_pair(make(inf))
    assert sim.n_inflow == 2
    U0np = state(sim)
    U0 = torch.from_numpy(U0np).cuda()
    theta = torch.tensor([inf2["p"], inf2["T"], inf2["vel"][0]], dtype=torch.float64, requires_grad=True)
    wts = torch.from_numpy(np.random.default_rng(5).standard_normal(U0np.shape)).cuda()
    nsteps = 8
    UN = rollout(sim, U0.clone(), theta, nsteps, 4)
    (UN * wts).sum().backward()

    sim2 = cases.build_gpu(make(inf2))
    load(sim2, U0np)
    dts = []
    for _ in range(nsteps):
        assert sim2.run(max_step=1) == 1
        dts.append(sim2.time()["dt"])
    assert np.array_equal(UN.detach().cpu().numpy(), state(sim2))

    def J_of(inflow):
        s = cases.build_gpu(make(inflow))
        X = U0
        for dt in dts:
            X = step_dt(s, X, dt)
        return float((X * wts).sum())

    for comp, key in ((0, "p"), (1, "T")):
        h = 1e-6 * inf2[key]
        fd = (J_of(dict(inf2, **{key: inf2[key] + h})) - J_of(dict(inf2, **{key: inf2[key] - h}))) / (2 * h)
        ad = float(theta.grad[comp])
        assert abs(fd - ad) <= 1e-4 * abs(fd), (key, fd, ad)


def test_step_chain_and_fused_step_adjoint():
    """gdfv_steps_dt equals repeated gdfv_step_dt bit for bit (states and predictor
    states), and gdfv_step_adjoint equals the predictor-corrector adjoint composed
    from two gdfv_residual_vjp products, inflow cotangents included."""
    from gdfv.autograd import step_adjoint, step_dt, steps_dt, vjp
    case = cases.c2_inflow_box(n=(24, 16, 12), noise_all=True)
    _, sim = cases.build_pair(case)
    U0 = torch.from_numpy(sim.get_conserved(0)).cuda()
    dts = [3.0e-7, 2.5e-7, 3.5e-7]
    outs = [torch.empty_like(U0) for _ in dts]
    preds = [torch.empty_like(U0) for _ in dts]
    steps_dt(sim, U0, dts, outs, preds)
    U = U0
    for m, dt in enumerate(dts):
        nxt, U1 = step_dt(sim, U, dt, with_predictor=True)
        assert torch.equal(nxt, outs[m]) and torch.equal(U1, preds[m])
        U = nxt
    rng = np.random.default_rng(11)
    lam0 = torch.from_numpy(rng.standard_normal(tuple(U0.shape))).cuda()
    dt = dts[0]
    a = lam0 * (0.5 * dt)
    mu, g1 = vjp(sim, preds[0], a)
    g0, g0i = vjp(sim, U0, a + mu * dt)
    want, want_in = lam0 + mu + g0, g1 + g0i
    lam = lam0.clone()
    gin = torch.zeros((sim.n_inflow, 6), dtype=torch.float64, device=lam.device)
    step_adjoint(sim, U0, preds[0], dt, lam, gin)
    torch.cuda.synchronize()
    assert torch.allclose(lam, want, rtol=1e-13, atol=1e-13 * float(want.abs().max()))
    assert np.allclose(gin.cpu().numpy(), want_in.numpy(), rtol=1e-12, atol=1e-12 * float(want_in.abs().max()))


def test_pipelined_rollout_adjoint_matches_sequential():
    """gdfv_rollout_adjoint (segment recomputation on a second stream overlapping the
    adjoint of the next segment) gives the lambda and inflow cotangents of the
    sequential gdfv_steps_dt + gdfv_step_adjoint composition (to the rounding of the
    FP64 atomic accumulation, whose order varies run to run)."""
    from gdfv._lib import check, ffi
    from gdfv.autograd import _p, step_adjoint, steps_dt
    case = cases.c2_inflow_box(n=(40, 24, 20), noise_all=True)
    _, sim = cases.build_pair(case)
    U0 = torch.from_numpy(sim.get_conserved(0)).cuda()
    K, nsteps = 4, 11
    rng = np.random.default_rng(21)
    dts = list(2.0e-7 * (1.0 + 0.2 * rng.random(nsteps)))
    ckpts, states = [U0.clone()], [U0.clone()]
    outs = [torch.empty_like(U0) for _ in range(nsteps)]
    preds = [torch.empty_like(U0) for _ in range(nsteps)]
    steps_dt(sim, U0, dts, outs, preds)
    for s in range(1, (nsteps + K - 1) // K):
        ckpts.append(outs[s * K - 1].clone())
    lam0 = torch.from_numpy(rng.standard_normal(tuple(U0.shape))).cuda()
    # sequential reference
    lam = lam0.clone()
    gin = torch.zeros((sim.n_inflow, 6), dtype=torch.float64, device=lam.device)
    for n in reversed(range(nsteps)):
        step_adjoint(sim, U0 if n == 0 else outs[n - 1], preds[n], dts[n], lam, gin)
    torch.cuda.synchronize()
    # pipelined
    for last_ready in (0, 1):
        lam2 = lam0.clone()
        gin2 = torch.zeros_like(gin)
        work = [torch.empty_like(U0) for _ in range(4 * K)]
        if last_ready:   # the last segment (steps 8..10) handed over as a forward pass keeps it
            s_last = (len(ckpts) - 1) * K
            for m in range(nsteps - s_last):
                work[K + m].copy_(preds[s_last + m])
                if s_last + m < nsteps - 1:
                    work[m].copy_(outs[s_last + m])
        pc = ffi.new("double*[]", [_p(t) for t in ckpts])
        pw = ffi.new("double*[]", [_p(t) for t in work])
        pd = ffi.new("double[]", dts)
        torch.cuda.synchronize()
        check(sim.ctx, sim.L.gdfv_rollout_adjoint(sim.ctx, pc, len(ckpts), pd, nsteps, K, pw, last_ready, _p(lam2),
                                                  _p(gin2)))
        torch.cuda.synchronize()
        assert torch.allclose(lam, lam2, rtol=1e-12, atol=1e-12 * float(lam.abs().max())), last_ready
        assert torch.allclose(gin, gin2, rtol=1e-12, atol=0.0), last_ready


def test_run_record_is_the_stepwise_trajectory():
    """gdfv_run_record (steps and their records on the device, one host round trip) keeps
    the states, predictor states and dts that gdfv_run taken one step at a time with
    gdfv_last_predictor_state gives, bit for bit; NULL entries keep nothing."""
    from gdfv._lib import check, ffi
    from gdfv.autograd import _p, _state_view
    case = cases.c2_inflow_box(n=(40, 24, 20), noise_all=True)
    _, sim = cases.build_pair(case)
    U0 = torch.from_numpy(sim.get_conserved(0)).cuda()
    nsteps = 7
    states = [torch.full_like(U0, -1.0) for _ in range(nsteps)]
    preds = [torch.full_like(U0, -1.0) for _ in range(nsteps)]
    keep = [n != 3 for n in range(nsteps)]   # step 3's state is not asked for
    sim.set_time(0.0, 0, sim.config.dt_init)
    _state_view(sim).copy_(U0)
    torch.cuda.synchronize()
    dts = ffi.new("double[]", nsteps)
    check(sim.ctx, sim.L.gdfv_run_record(sim.ctx, nsteps, ffi.new("double*[]", [_p(t) if k else ffi.NULL
                                                                                  for t, k in zip(states, keep)]),
                                         ffi.new("double*[]", [_p(t) for t in preds]), dts))
    UN = _state_view(sim).clone()
    sim.set_time(0.0, 0, sim.config.dt_init)
    _state_view(sim).copy_(U0)
    torch.cuda.synchronize()
    prev = U0.clone()
    for n in range(nsteps):
        assert sim.run(max_step=1) == 1
        assert sim.time()["dt"] == dts[n]
        pred = torch.empty_like(U0)
        check(sim.ctx, sim.L.gdfv_last_predictor_state(sim.ctx, _p(prev), _p(pred)))
        cur = _state_view(sim).clone()
        torch.cuda.synchronize()
        assert torch.equal(pred, preds[n]), n
        if keep[n]:
            assert torch.equal(cur, states[n]), n
        else:
            assert bool((states[n] == -1.0).all())
        prev = cur
    assert torch.equal(prev, UN)


def test_resident_trajectory_rollout_matches_checkpointed():
    """rollout's default keeps the whole trajectory on the device when it fits (one
    segment, nothing recomputed); its gradients equal those of the checkpointed form (a
    checkpoint every 4 steps, segments recomputed) to the rounding of the FP64 atomic
    accumulation."""
    from gdfv.autograd import resident_steps, rollout
    case = cases.c2_inflow_box(n=(40, 24, 20), noise_all=True)
    inf = cases.inflow_state_m3()
    _, sim = cases.build_pair(case)
    U0 = torch.from_numpy(sim.get_conserved(0)).cuda()
    nsteps = 11
    assert resident_steps(sim, nsteps) == nsteps
    grads = []
    for K in (None, 4):
        theta = torch.tensor([inf["p"], inf["T"], inf["vel"][0]], dtype=torch.float64, requires_grad=True)
        U0r = U0.clone().requires_grad_(True)
        UN = rollout(sim, U0r, theta, nsteps, K)
        wall_pressure(case, UN, case.R).backward()
        grads.append((U0r.grad.clone(), theta.grad.clone()))
    (gr, tr), (gc, tc) = grads
    assert torch.allclose(gr, gc, rtol=1e-11, atol=1e-11 * float(gc.abs().max()))
    assert torch.allclose(tr, tc, rtol=1e-11, atol=0.0)


@pytest.mark.parametrize("case_name", ["inflow", "multiblock"])
def test_frechet_jvp_matches_oracle(case_name):
    """gdfv_residual_jvp against the oracle's restatement of evalJacobianVecProd
    (e4/steadystate_core.d:1878-1970): bit for bit with a given sigma and with the
    GPU's Knoll-McHugh sigma (whose device reduction may round differently from the
    oracle's sequential sum: checked to 1e-13), with and without a supplied R(U)."""
    from gdfv.autograd import jvp, residual_eval
    case = (cases.c2_inflow_box(n=(24, 16, 12)) if case_name == "inflow"
            else cases.multiblock_lattice(nb=(2, 1, 2), sizes=(16, 24), seed=3))
    orc, sim, U = _state_after(case, 4)
    rng = np.random.default_rng(8)
    v = rng.standard_normal(U.shape) * np.abs(U).max(axis=1, keepdims=True)
    Ut, vt = torch.from_numpy(U).cuda(), torch.from_numpy(v).cuda()
    Uo, vo = _gpu_to_oracle_layout(case, U), _gpu_to_oracle_layout(case, v)
    Jv_o, sig_o = orc.jvp_real(Uo, vo)
    Jv_g, sig_g = jvp(sim, Ut, vt)
    assert abs(sig_g - sig_o) <= 1e-13 * sig_o
    Jv_o2, _ = orc.jvp_real(Uo, vo, sigma=sig_g)
    assert np.array_equal(_gpu_to_oracle_layout(case, Jv_g.cpu().numpy()), Jv_o2)
    R0 = residual_eval(sim, Ut)
    Jv_g2, _ = jvp(sim, Ut, vt, R0=R0, sigma=sig_g)
    assert torch.equal(Jv_g, Jv_g2)


@pytest.mark.parametrize("case_name", ["mhd", "mhd_slip_dipole", "hllc", "graded"])
def test_frechet_jvp_more_forms_match_oracle(case_name):
    """gdfv_residual_jvp bit for bit against the oracle's evalJacobianVecProd at a given
    sigma on the other forms of the path: MHD (hlle + GLM on Orszag-Tang, and slip walls
    with the dipole ghosts; both sides take the same 4 steps first, so that they hold the
    same c_h), hllc and a graded block."""
    from gdfv.autograd import jvp
    case = {"mhd": lambda: cases.orszag_tang(n=(32, 32, 4)),
            "mhd_slip_dipole": lambda: cases.mhd_slip_dipole(n=(32, 24, 4)),
            "hllc": lambda: cases.c2_inflow_box(n=(24, 16, 12), flux="hllc", noise_all=True),
            "graded": lambda: cases.graded_inflow_box()}[case_name]()
    orc, sim = cases.build_pair(case)
    assert orc.run(4) == 0 and sim.run(max_step=4) == 4
    U = np.concatenate([sim.get_conserved(b) for b in range(len(case.blocks))], axis=1)
    for b in range(len(case.blocks)):
        assert orc.set_U(b, sim.get_conserved(b)) == 0
    rng = np.random.default_rng(15)
    v = rng.standard_normal(U.shape) * (np.abs(U).max(axis=1, keepdims=True) + 1e-30)
    Ut, vt = torch.from_numpy(U).cuda(), torch.from_numpy(v).cuda()
    Uo, vo = _gpu_to_oracle_layout(case, U), _gpu_to_oracle_layout(case, v)
    Jv_g, sig_g = jvp(sim, Ut, vt)
    Jv_o, _ = orc.jvp_real(Uo, vo, sigma=sig_g)
    assert np.array_equal(_gpu_to_oracle_layout(case, Jv_g.cpu().numpy()), Jv_o)


def test_vjp_run_to_run_variation_is_bounded():
    """The VJP scatters the stencil cotangents with FP64 atomic additions, whose order
    varies from run to run: repeated products of the same (U, W) agree to a stated bound
    -- 1e-13 relative to the largest cotangent of each conserved quantity -- and the
    rollout gradient dJ/dU0 of a 10-step rollout likewise (the order of the additions
    changes only the last bits)."""
    from gdfv.autograd import rollout, vjp
    case = cases.c2_inflow_box(n=(48, 40, 36), noise_all=True)
    orc, sim, U = _state_after(case, 4)
    Ut = torch.from_numpy(U).cuda()
    W = torch.from_numpy(np.random.default_rng(9).standard_normal(U.shape)).cuda()
    Gs = [vjp(sim, Ut, W)[0].cpu().numpy() for _ in range(4)]
    for G in Gs[1:]:
        scale = np.abs(Gs[0]).max(axis=1, keepdims=True)
        assert np.max(np.abs(G - Gs[0]) / scale) <= 1e-13
    inf = cases.inflow_state_m3()
    grads = []
    U0np = sim.get_conserved(0)
    for _ in range(2):
        U0 = torch.from_numpy(U0np.copy()).cuda().requires_grad_(True)
        theta = torch.tensor([inf["p"], inf["T"], inf["vel"][0]], dtype=torch.float64, requires_grad=True)
        UN = rollout(sim, U0, theta, 10, 5)
        (UN * W).sum().backward()
        grads.append(U0.grad.cpu().numpy())
    scale = np.abs(grads[0]).max(axis=1, keepdims=True)
    assert np.max(np.abs(grads[1] - grads[0]) / scale) <= 1e-12
