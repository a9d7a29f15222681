"""The CPU oracle pinned against the reference (CPU only, no GPU needed).

* the reference's own integration-test answers (tests/golden/reference_job_answers.json):
  examples/eilmer/3D/sod-shock-tube/sg/sod-test.rb and
  examples/eilmer/2D/MHDShockTube/MHD-ShockTube-Test.rb;
* the reference's 2D Euler method-of-manufactured-solutions smoke test
  (examples/eilmer/2D/manufactured-solution/sg/smoke-tests/mms-euler-test.rb): steps
  to t = 60 ms and the density error norms, which pin the Eilmer-4 branches that the
  chicken golden switches off (entropy fix, face-frame velocity, the cell-centre sound
  speed kept through the rhou update, predictor-corrector);
* the reference's own compiled chicken solver: a golden run committed in
  tests/golden/chicken_lattice.npz (made by tests/golden/make_golden.py), and a
  live run when oracle/_ref/chkn-run has been built here;
* the ExchangeBC_FullFace ghost map of every face pair and orientation, read from the
  reference's source (tests/golden/exchange_map.json, made by
  tests/golden/make_exchange_map.py), and the rotation of the ghosts' vectors against
  the flow it stands for (a quarter domain against the whole).
"""
import json
import os

import numpy as np
import pytest

import cases

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def answers():
    with open(os.path.join(GOLDEN, "reference_job_answers.json")) as f:
        return json.load(f)


def test_sod_reference_answers():
    a = answers()["sod"]
    orc = cases.build_oracle(cases.sod_eilmer())
    assert orc.run(600, max_time=a["max_time"]) == 0
    assert abs(orc.time()["step"] - a["steps"]) < a["steps_tol"]
    fl = orc.get_flow(0)
    for x, probe in ((0.78, a["probe_078"]), (0.6, a["probe_060"])):
        c = int(x / 0.01)
        got = {"rho": fl["rho"][c], "p": fl["p"][c], "T": fl["T"][c], "velx": fl["vx"][c]}
        for k, ref in probe.items():
            assert abs(got[k] - ref) / ref < a["rel_tol"], (x, k, got[k], ref)


def test_mhd_shock_tube_reference_answers():
    a = answers()["mhd_shock_tube"]
    orc = cases.build_oracle(cases.mhd_shock_tube())
    assert orc.run(100000, max_time=a["max_time"]) == 0
    assert abs(orc.time()["step"] - a["steps"]) < a["steps_tol"]
    nic, dx, s4 = 256, 0.5 / 256, np.sqrt(4 * np.pi)
    for r, xp in enumerate((0.3, 0.5, 0.7)):
        blk = 0 if xp < 0.5 else 1
        fl = orc.get_flow(blk)
        i = min(int((xp - 0.5 * blk) / dx), nic - 1)
        c = i + nic * 1
        got = {"p": fl["p"][c], "vel.y": fl["vy"][c], "vel.z": fl["vz"][c], "B.y": fl["By"][c] * s4,
               "B.z": fl["Bz"][c] * s4, "rho": fl["rho"][c]}
        for k, tol in a["tol"].items():
            assert abs(got[k] - a[k][r]) < tol, (xp, k, got[k], a[k][r])


def _oracle_for_chicken_job(job, dt, nsteps):
    from oracle import OracleSim
    s = OracleSim(flux_calculator="ausmdv", gasdynamic_update_scheme="tvd_rk3", chicken_compat=1,
                  apply_entropy_fix=0, extrema_clipping=0, R=287.1, gamma=1.4)
    blocks = list(job.blocks())
    index = {b: n for n, b in enumerate(blocks)}
    for b in blocks:
        s.add_block(job.nics[b[0]], job.njcs[b[1]], job.nkcs[b[2]], job.d, job.d, job.d, *job.origin(*b))
    pairs = {"iminus": ("west", 0, -1), "iplus": ("east", 0, 1), "jminus": ("south", 1, -1),
             "jplus": ("north", 1, 1), "kminus": ("bottom", 2, -1), "kplus": ("top", 2, 1)}
    opposite = {"west": "east", "east": "west", "south": "north", "north": "south", "bottom": "top", "top": "bottom"}
    nb = (job.nib, job.njb, job.nkb)
    for b in blocks:
        for cf, (face, axis, step) in pairs.items():
            tag = job.bcs.get((b, cf), "wall_with_slip")
            if tag == "inflow":
                p, T, vel = job.inflow
                s.set_bc(index[b], face, "inflow_supersonic", inflow=dict(p=p, T=T, vel=vel))
            elif tag == "outflow":
                s.set_bc(index[b], face, "extrapolate")
            elif tag == "exchange":
                o = list(b)
                o[axis] = (o[axis] + step) % nb[axis]
                s.set_bc(index[b], face, "exchange", other_block=index[tuple(o)], other_face=opposite[face])
            else:
                s.set_bc(index[b], face, "wall_with_slip")
    for b in blocks:
        rho, vel, T = job.flow[b]
        s.set_flow_rhoT(index[b], rho, vel, T)
    s.init()
    assert s.run(nsteps, fixed_dt=dt) == 0
    return s, index


def _compare_with_chicken(s, index, flows, tol):
    for b, fc in flows.items():
        fo = s.get_flow(index[b])
        for key, ck in (("rho", "rho"), ("vx", "velx"), ("vy", "vely"), ("vz", "velz"), ("p", "p"), ("T", "T")):
            ref = fc[ck]
            scale = np.max(np.abs(ref))
            assert np.max(np.abs(fo[key] - ref)) <= tol * scale, (b, key)


def test_oracle_matches_chicken_golden():
    """Oracle in chicken-compatible mode vs the committed chicken run (1e-12 of each field's scale)."""
    import sys
    sys.path.insert(0, GOLDEN)
    import make_golden
    job = make_golden.chicken_lattice_job()
    data = np.load(os.path.join(GOLDEN, "chicken_lattice.npz"))
    for b in job.blocks():  # the fixture carries its own initial density field
        rho, vel, T = job.flow[b]
        job.flow[b] = (data[f"init_b{b[0]}{b[1]}{b[2]}_rho"].reshape(np.shape(rho)), vel, T)
    flows = {b: {k: data[f"b{b[0]}{b[1]}{b[2]}_{k}"] for k in ("rho", "velx", "vely", "velz", "p", "T")}
             for b in job.blocks()}
    s, index = _oracle_for_chicken_job(job, make_golden.DT, make_golden.NSTEPS)
    _compare_with_chicken(s, index, flows, 1e-12)


def test_oracle_matches_chicken_live_periodic():
    """A live chicken run (when built here): 2x2x1 lattice, periodic exchange in j and k,
    slip walls on the i faces (chicken mirrors cell 0 into both ghost layers)."""
    import chicken_job as cj
    if not cj.available():
        pytest.skip("oracle/_ref/chkn-run not built")
    d = 1.0 / 1024
    job = cj.LatticeJob([8, 8], [4, 4], [4], d)
    rng = np.random.default_rng(5)
    for b in job.blocks():
        shp = (4, 4, 8)
        x = (np.arange(8) + 0.5 + 8 * b[0])[None, None, :]
        p_like = np.where(x < 8, 1.0e5, 1.0e4) * np.ones(shp)
        rho = p_like / (cj.R * 300.0) * (1 + 0.01 * rng.standard_normal(shp))
        job.flow[b] = (rho, (10.0 * rng.standard_normal(shp), 0.0, 0.0), 300.0)
        job.bcs[(b, "jminus")] = "exchange"
        job.bcs[(b, "jplus")] = "exchange"
        job.bcs[(b, "kminus")] = "exchange"
        job.bcs[(b, "kplus")] = "exchange"
        job.bcs[(b, "iminus" if b[0] == 1 else "iplus")] = "exchange"
    flows, _, _ = cj.run(job, 1.0e-8, 15)
    s, index = _oracle_for_chicken_job(job, 1.0e-8, 15)
    _compare_with_chicken(s, index, flows, 1e-12)


def mms_euler_oracle():
    """examples/eilmer/2D/manufactured-solution/sg/smoke-tests with case-euler.txt
    (mms.lua, case 1): 2D, 16 x 16 cells on the unit square as 2 x 2 blocks of 8 x 8
    (FBArray nib = njb = 2, full-face exchange inside), ausmdv, interpolation order 2
    with limiter and extrema clipping off, predictor-corrector, stringent CFL 0.5,
    dt_init 1e-6, ideal gas R = 287, gamma = 1.4; initial state p = 1e5, T = p/R,
    vel = (800, 800); west and south faces: ghost cells from the manufactured solution
    (UserDefinedBC), north and east: OutFlowBC_SimpleExtrapolate xOrder 1; the
    manufactured source terms in every cell.  Fields from tests/golden/mms_euler_16.npz
    (tests/golden/make_mms.py)."""
    from oracle import OracleSim
    g = np.load(os.path.join(GOLDEN, "mms_euler_16.npz"))
    R, gamma = float(g["R"]), float(g["gamma"])
    s = OracleSim(R=R, gamma=gamma, flux_calculator="ausmdv", dimensions=2, apply_limiter=0, extrema_clipping=0,
                  stringent_cfl=1, cfl_value=0.5, dt_init=1.0e-6)
    n, h = 8, 1.0 / 16
    for bj in range(2):
        for bi in range(2):
            s.add_block(n, n, 1, h, h, 1.0, 0.5 * bi, 0.5 * bj, 0.0)
    idx = lambda bi, bj: bi + 2 * bj
    for bj in range(2):
        for bi in range(2):
            b = idx(bi, bj)
            if bi == 0:
                s.set_ghost_states(b, "west", g["ghost_west"][:, None, bj * n:(bj + 1) * n, :])
            else:
                s.set_bc(b, "west", "exchange", other_block=idx(0, bj), other_face="east")
            if bi == 1:
                s.set_bc(b, "east", "extrapolate", x_order=1)
            else:
                s.set_bc(b, "east", "exchange", other_block=idx(1, bj), other_face="west")
            if bj == 0:
                s.set_ghost_states(b, "south", g["ghost_south"][:, bi * n:(bi + 1) * n, None, :])
            else:
                s.set_bc(b, "south", "exchange", other_block=idx(bi, 0), other_face="north")
            if bj == 1:
                s.set_bc(b, "north", "extrapolate", x_order=1)
            else:
                s.set_bc(b, "north", "exchange", other_block=idx(bi, 1), other_face="south")
            p0 = 1.0e5
            T0 = p0 / R
            s.set_flow_rhoT(b, p0 / (T0 * R), (800.0, 800.0, 0.0), T0)
            Q = g["Q"][:, bj * n:(bj + 1) * n, bi * n:(bi + 1) * n].reshape(5, n * n)
            s.set_source(b, Q)
    s.init()
    return s, g


def test_oracle_e4_mode_pinned_by_mms_euler():
    """mms-euler-test.rb: 2620 +/- 3 steps to t = 60 ms, and the volume-weighted norms of
    the density error against the manufactured solution (flowsolution.d:305-345:
    L1 = sum V|e| / sum V, L2 = sqrt(sum V e^2 / sum V), Linf = max |e|) within a
    relative 1e-3 of L1 = 5.992287970340e-04, L2 = 8.134693405237e-04,
    Linf = 2.746228919538e-03 (mms-euler-test.rb:38, :47-62).  The oracle takes exactly
    2620 steps and meets the three norms to about 1e-11 relative (the reference prints
    13 significant digits); asserted at 1e-9 as well as at the reference's 1e-3."""
    s, g = mms_euler_oracle()
    assert s.run(100000, max_time=60.0e-3) == 0, s.last_error()
    steps = s.time()["step"]
    assert abs(steps - 2620) < 3, steps
    assert steps == 2620
    n = 8
    err = np.zeros((16, 16))
    for bj in range(2):
        for bi in range(2):
            rho = s.get_flow(bi + 2 * bj)["rho"].reshape(n, n)
            err[bj * n:(bj + 1) * n, bi * n:(bi + 1) * n] = rho - g["rho_exact"][bj * n:(bj + 1) * n, bi * n:(bi + 1) * n]
    norms = {"L1": np.mean(np.abs(err)), "L2": np.sqrt(np.mean(err ** 2)), "Linf": np.max(np.abs(err))}
    refs = {"L1": 5.992287970340e-04, "L2": 8.134693405237e-04, "Linf": 2.746228919538e-03}
    for k, ref in refs.items():
        assert abs(norms[k] - ref) / ref < 1.0e-3, (k, norms[k], ref, steps)
        assert abs(norms[k] - ref) / ref < 1.0e-9, (k, norms[k], ref)


def test_oracle_graded_block_with_uniform_spacing_is_the_uniform_block():
    """A graded (rectilinear) block whose vertices are evenly spaced -- at 1/1024 m, so the
    cell lengths are exact -- computes the uniform block's results bit for bit: the
    per-face l2r2 weights, areas, volumes and signal lengths of the graded path reduce to
    the uniform ones."""
    cu = cases.c2_inflow_box(n=(24, 16, 12), seed=17, d=1 / 1024.0)
    cg = cases.graded_inflow_box(n=(24, 16, 12), uniform=True)
    ou, og = cases.build_oracle(cu), cases.build_oracle(cg)
    U = ou.get_U(0)
    assert ou.set_U(0, U) == 0 and og.set_U(0, U) == 0
    assert ou.run(6) == 0 and og.run(6) == 0
    assert np.array_equal(ou.get_U(0), og.get_U(0))
    assert ou.time()["dt"] == og.time()["dt"]


def exchange_maps():
    with open(os.path.join(GOLDEN, "exchange_map.json")) as f:
        return json.load(f)["maps"]


def exchange_ghosts(rec):
    """Every ghost of a map's face on small blocks (3 x 4 x 5 cells, 3 x 4 x 1 in 2D; the
    partner sized as the map needs) with the partner cell the reference's map names."""
    dims, f, src = rec["dims"], rec["face"], rec["src"]
    n = [3, 4, 5] if dims == 3 else [3, 4, 1]
    on = [6 if sel == 3 else n[sel] for sel, _ in src]
    ax = f // 2
    t = [d for d in range(3) if d != ax]
    for m in range(2):
        for a in range(n[t[0]]):
            for b in range(n[t[1]]):
                ijk = [0, 0, 0]
                ijk[t[0]], ijk[t[1]] = a, b
                ijk[ax] = n[ax] + m if f & 1 else -1 - m
                want = tuple(on[d] - 1 - (m if sel == 3 else ijk[sel]) if flip else (m if sel == 3 else ijk[sel])
                             for d, (sel, flip) in enumerate(src))
                yield n, on, ijk, want


def test_oracle_exchange_map_is_the_reference_map():
    """full_face_copy.d:680-1409 spells out the ghost-to-source map for 4 x 4 face pairs
    in 2D and 6 x 6 pairs x 4 orientations in 3D; the oracle restates it as one rule.
    Every ghost of every case agrees."""
    import oracle
    maps = exchange_maps()
    assert len(maps) == 160
    for rec in maps:
        for n, on, ijk, want in exchange_ghosts(rec):
            got = oracle.exchange_source(rec["dims"], rec["face"], rec["other_face"], rec["orientation"], n, on, ijk)
            assert got == want, (rec, ijk)
    # a ghost two layers out, and a partner too small for the map
    assert oracle.exchange_source(3, 1, 3, 0, [3, 4, 5], [4, 6, 5], [5, 0, 0]) is None
    assert oracle.exchange_source(3, 1, 3, 1, [3, 4, 5], [4, 6, 5], [3, 3, 4]) is None


def test_oracle_rotational_exchange_is_the_whole_domain():
    """A flow with four-fold rotational symmetry on the quadrant x, y >= 0, its x = 0 and
    y = 0 faces joined by exchanges that turn the ghosts' velocity by +-90 degrees
    (reorient_vector_quantities, flowstate.d:393-400), against the same flow on the whole
    square: after 40 steps (the momentum changes by O(1) relative to its maximum) the
    quadrant agrees to rounding; without the rotation it does not."""
    q, f = cases.quarter_rotational(n=(16, 16, 2)), cases.full_rotational(n=(16, 16, 2))
    for c in (q, f):
        c.config.update(dt_init=4e-7, dt_max=4e-7)
    oq, of = cases.build_oracle(q), cases.build_oracle(f)
    U0 = of.get_U(0).reshape(5, 2, 32, 32)[:, :, 16:, 16:].copy()
    assert oq.run(40) == 0 and of.run(40) == 0
    Uq = oq.get_U(0).reshape(5, 2, 16, 16)
    Uf = of.get_U(0).reshape(5, 2, 32, 32)[:, :, 16:, 16:]
    for qv in (0, 1, 2, 4):   # z momentum stays 0
        scale = np.max(np.abs(Uf[qv]))
        assert np.max(np.abs(Uq[qv] - Uf[qv])) <= 1e-13 * scale, qv
    assert np.max(np.abs(Uf[1] - U0[1])) >= 0.5 * np.max(np.abs(Uf[1]))
    plain = cases.quarter_rotational(n=(16, 16, 2))
    plain.config.update(dt_init=4e-7, dt_max=4e-7)
    for face in ("west", "south"):
        plain.blocks[0]["bcs"][face][1].pop("Rmatrix")
    op = cases.build_oracle(plain)
    assert op.run(40) == 0
    Up = op.get_U(0).reshape(5, 2, 16, 16)
    assert np.max(np.abs(Up[1] - Uf[1])) >= 0.1 * np.max(np.abs(Uf[1]))

