"""The CPU oracle pinned against the reference (CPU only, no GPU needed).

* the reference's own integration-test answers (tests/golden/reference_job_answers.json):
  examples/eilmer/3D/sod-shock-tube/sg/sod-test.rb and
  examples/eilmer/2D/MHDShockTube/MHD-ShockTube-Test.rb;
* the reference's own compiled chicken solver: a golden run committed in
  tests/golden/chicken_lattice.npz (made by tests/golden/make_golden.py), and a
  live run when oracle/_ref/chkn-run has been built here.
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
