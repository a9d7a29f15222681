"""chicken job directories through the GPU path (gdfv.chicken).

Jobs are written in chicken's own formats (config.json, binary or gzipped grid and
flow files, times.data) by the test infrastructure in oracle/chicken_job.py; the
loader must reproduce the blocks, boundary tags and initial state, the GPU run of a
loaded job must match the oracle run of the same case, and flow files written
back must read as chicken reads them.
"""
import gzip
import os
import sys

import numpy as np
import pytest

import cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import chicken_job as cj  # noqa: E402

from gdfv import chicken  # noqa: E402


def lattice_job(seed=3):
    """2 x 2 x 1 lattice: M=3 inflow on i-minus, outflow on i-plus, exchange inside,
    periodic exchange across the k faces, slip walls on the j edges."""
    d = 1.0 / 1024
    job = cj.LatticeJob([16, 8], [8, 12], [6], d)
    T = 220.0
    u = 3.0 * np.sqrt(cj.GAMMA * cj.R * T)
    job.inflow = (5.0e3, T, (u, 0.0, 0.0))
    rng = np.random.default_rng(seed)
    rho_inf = 5.0e3 / (cj.R * T)
    for b in job.blocks():
        shp = (job.nkcs[b[2]], job.njcs[b[1]], job.nics[b[0]])
        job.flow[b] = (rho_inf * (1 + 0.01 * rng.standard_normal(shp)), (u, 0.0, 0.0), T)
        i, j, k = b
        job.bcs[(b, "iminus")] = "inflow" if i == 0 else "exchange"
        job.bcs[(b, "iplus")] = "outflow" if i == 1 else "exchange"
        if j == 1:
            job.bcs[(b, "jminus")] = "exchange"
        if j == 0:
            job.bcs[(b, "jplus")] = "exchange"
        job.bcs[(b, "kminus")] = "exchange"
        job.bcs[(b, "kplus")] = "exchange"
    return job


def equivalent_case(job, precision="fp64"):
    """The same problem as a test case (for the oracle and the directly built GPU path)."""
    c = cases.Case("chicken_lattice", dict(flux_calculator="ausmdv", flux_precision=precision, dt_init=2e-7,
                                            dt_max=1e-3, cfl_value=0.5), cj.R, cj.GAMMA)
    order = sorted(job.blocks(), key=lambda b: (b[2], b[1], b[0]))
    idx = {b: n for n, b in enumerate(order)}
    p, T, vel = job.inflow
    inf = dict(p=p, T=T, vel=vel)
    face_name = {"iminus": "west", "iplus": "east", "jminus": "south", "jplus": "north", "kminus": "bottom",
                 "kplus": "top"}
    opp = {"iminus": "east", "iplus": "west", "jminus": "north", "jplus": "south", "kminus": "top", "kplus": "bottom"}
    nb = (job.nib, job.njb, job.nkb)
    for b in order:
        bcs = {}
        for f in cj.FACES:
            tag = job.bcs.get((b, f), "wall_with_slip")
            if tag == "exchange":
                axis = cj.FACES.index(f) // 2
                o = list(b)
                o[axis] = (o[axis] + (1 if f.endswith("plus") else -1)) % nb[axis]
                bcs[face_name[f]] = ("exchange_over_full_face", dict(other=idx[tuple(o)], other_face=opp[f]))
            elif tag == "inflow":
                bcs[face_name[f]] = ("inflow_supersonic", dict(inflow=inf))
            elif tag == "outflow":
                bcs[face_name[f]] = ("outflow_simple_extrapolate", dict(x_order=0))
        rho, v, Tb = job.flow[b]
        n = (job.nics[b[0]], job.njcs[b[1]], job.nkcs[b[2]])
        c.add_block(n, (job.d,) * 3, job.origin(*b), bcs, rho, v, Tb)
    return c


def test_parse_job_binary_and_text(tmp_path):
    job = lattice_job()
    d = str(tmp_path / "job")
    job.write(d, 2e-7, 10)
    cj_parsed = chicken.ChickenJob(d)
    assert cj_parsed.binary
    assert cj_parsed.active_blocks() == [(0, 0, 0), (1, 0, 0), (0, 1, 0), (1, 1, 0)]
    assert cj_parsed.neighbour((1, 0, 0), "iplus") == (0, 0, 0)          # periodic wrap
    assert cj_parsed.neighbour((0, 0, 0), "kminus") == (0, 0, 0)
    for b in cj_parsed.active_blocks():
        nic, njc, nkc = cj_parsed.shape(b)
        gpath = os.path.join(d, "grid", f"grid-{b[0]:04d}-{b[1]:04d}-{b[2]:04d}.bin")
        dxyz, origin = chicken.uniform_geometry(chicken.read_grid(gpath, nic, njc, nkc))
        assert np.allclose(dxyz, job.d) and np.allclose(origin, job.origin(*b))
        fpath = os.path.join(d, "flow", "t0000", f"flow-{b[0]:04d}-{b[1]:04d}-{b[2]:04d}.bin")
        fl = chicken.read_flow(fpath, nic * njc * nkc, cj_parsed.iovars)
        assert np.array_equal(fl["rho"], np.broadcast_to(job.flow[b][0], (nkc, njc, nic)).ravel())
        # the same data as gzipped text files (chicken's other format) read the same
        gz = gpath[:-4] + ".gz"
        verts = chicken.read_grid(gpath, nic, njc, nkc)
        with gzip.open(gz, "wt") as f:
            f.write(f"structured_grid 1.0\nlabel: \ndimensions: 3\nniv: {nic + 1}\nnjv: {njc + 1}\nnkv: {nkc + 1}\n")
            f.write("\n".join(" ".join(repr(float(v)) for v in p) for p in verts.reshape(-1, 3)) + "\n")
        assert np.array_equal(chicken.read_grid(gz, nic, njc, nkc), verts)
    with pytest.raises(ValueError):
        chicken.uniform_geometry(np.random.default_rng(0).random((3, 3, 3, 3)))


@pytest.mark.gpu
def test_loaded_job_matches_oracle_and_writes_back(tmp_path):
    job = lattice_job()
    d = str(tmp_path / "job")
    job.write(d, 2e-7, 10)
    sim, cjob = chicken.load_job(d, dt_init=2e-7)
    case = equivalent_case(job)
    orc, _ = cases.build_pair(case)
    # both start from the flow file's (rho, T, vel); the oracle encodes and decodes it
    for bi in range(len(case.blocks)):
        sim.set_conserved(bi, orc.get_U(bi))
    assert orc.run(6) == 0
    assert sim.run(max_step=6) == 6
    for bi in range(len(case.blocks)):
        errs = cases.cell_errors(sim.get_conserved(bi), orc.get_U(bi), False)
        assert max(errs.values()) <= 1e-12, (bi, errs)
    chicken.write_flow(sim, cjob, 1)
    back = job.read(d)   # chicken's reader (test infrastructure)
    for b, bi in cjob.index.items():
        U = sim.get_conserved(bi)
        assert np.allclose(back[b]["rho"], U[0], rtol=1e-15, atol=0)
        assert np.allclose(back[b]["velx"], U[1] / U[0], rtol=1e-14, atol=0)
    with open(os.path.join(d, "times.data")) as f:
        assert f.read().split()[-2] == "1"


# ---------------------------------------------------------------- the reference's own job
FFS = os.path.join(ROOT, "tests", "golden", "ffs_job")
FACE_NAMES = {"iminus": "west", "iplus": "east", "jminus": "south", "jplus": "north", "kminus": "bottom",
              "kplus": "top"}
OPPOSITE = {"west": "east", "east": "west", "south": "north", "north": "south", "bottom": "top", "top": "bottom"}


def oracle_from_job(jobdir, chicken_mode):
    """The oracle set up from a chicken job directory as gdfv.chicken.load_job reads it:
    active blocks with their grid's spacing and origin, face tags (missing tags are slip
    walls), the tagged inflow states and the flow file's rho, T and velocity.
    chicken_mode: chicken's own scheme (TVD-RK3, global-frame velocity, no clipping or
    entropy fix, recomputed sound speed, chicken's dt rule); else the Eilmer-4 options
    the GPU path computes with."""
    from oracle import OracleSim
    job = chicken.ChickenJob(jobdir)
    cfg = job.cfg
    opts = dict(flux_calculator="ausmdv", R=job.R, gamma=job.gamma, cfl_value=float(cfg["cfl_values"][0]),
                dt_init=float(cfg.get("dt_init", 1e-6)), cfl_count=int(cfg.get("cfl_count", 10)))
    if chicken_mode:
        opts.update(gasdynamic_update_scheme="tvd_rk3", chicken_compat=1, apply_entropy_fix=0, extrema_clipping=0)
    s = OracleSim(**opts)
    blocks = job.active_blocks()
    index = {b: n for n, b in enumerate(blocks)}
    geom = {}
    for b in blocks:
        nic, njc, nkc = job.shape(b)
        path = os.path.join(jobdir, "grid", f"grid-{b[0]:04d}-{b[1]:04d}-{b[2]:04d}.gz")
        d, origin = chicken.uniform_geometry(chicken.read_grid(path, nic, njc, nkc), path)
        geom[b] = (d, origin)
        s.add_block(nic, njc, nkc, *d, *origin)
    for b in blocks:
        for face in chicken.FACES:
            bc = job.blocks[b]["bcs"].get(face, {"tag": "wall_with_slip"})
            name = FACE_NAMES[face]
            if bc["tag"] == "exchange":
                s.set_bc(index[b], name, "exchange", other_block=index[job.neighbour(b, face)],
                         other_face=OPPOSITE[name])
            elif bc["tag"] == "inflow":
                fs = job.flow_states[bc["flow_state_index"]]
                s.set_bc(index[b], name, "inflow_supersonic", inflow=dict(p=fs["p"], T=fs["T"], vel=fs["vel"]))
            elif bc["tag"] == "outflow":
                s.set_bc(index[b], name, "extrapolate")
            else:
                assert bc["tag"] == "wall_with_slip", bc
                s.set_bc(index[b], name, "wall_with_slip")
    for b in blocks:
        nic, njc, nkc = job.shape(b)
        fl = chicken.read_flow(os.path.join(jobdir, "flow", "t0000", f"flow-{b[0]:04d}-{b[1]:04d}-{b[2]:04d}.gz"),
                               nic * njc * nkc, job.iovars)
        shp = (nkc, njc, nic)
        s.set_flow_rhoT(index[b], fl["rho"].reshape(shp), tuple(fl[v].reshape(shp) for v in ("velx", "vely", "velz")),
                        fl["T"].reshape(shp))
    s.init()
    return s, job, index, geom


def shock_position(p, x):
    """examples/chicken/test_chicken.py:45-71: along the bottom row of block (0,0,0), the
    first cell whose pressure exceeds the freestream by 1%, and the position where the
    pressure, interpolated linearly from the cell before, reaches the normal-shock value
    1047025 Pa; returns (position, one cell width)."""
    p0 = p[0]
    idx = int(np.argmax(p > p0 + 0.01 * p0))
    assert idx != 0
    xp, pp, xs, ps = x[idx - 1], p[idx - 1], x[idx], p[idx]
    pn = 1047025.00
    return (xs - xp) / (ps - pp) * (pn - pp) + xp, xs - xp


FFS_SHOCK_X = 0.41369441539674984   # examples/chicken/test_chicken.py:70


def test_ffs_job_shock_position_chicken_scheme():
    """The reference's forward-facing-step job (prepared by its own chkn_prep.py, inactive
    blocks below the step, slip walls by default) through the oracle in chicken's scheme
    and dt rule to t = 1 ms: the shock stands where test_chicken.py asserts it, within
    its tolerance of a tenth of a cell."""
    s, job, index, geom = oracle_from_job(FFS, chicken_mode=True)
    assert len(index) == 21 and len(job.blocks) == 25
    assert s.run(job.cfg["max_step"], max_time=job.cfg["max_time"]) == 0
    nic, njc, nkc = job.shape((0, 0, 0))
    p = s.get_flow(index[(0, 0, 0)])["p"].reshape(nkc, njc, nic)[0, 0, :]
    (dx, _, _), (x0, _, _) = geom[(0, 0, 0)]
    x = x0 + (np.arange(nic) + 0.5) * dx
    xn, cell = shock_position(p, x)
    assert abs(xn - FFS_SHOCK_X) < 0.1 * cell, (xn, FFS_SHOCK_X, s.time())


def test_ffs_job_oracle_matches_live_chicken(tmp_path):
    """The same job run by the reference's compiled chicken (CPU build, when present here)
    for 25 steps -- through two dt checks -- against the oracle in chicken's scheme:
    every block, every field to 1e-12 of the field's scale (the grid files' vertices
    differ from uniform spacing in the last bits)."""
    import shutil
    import subprocess
    if not cj.available():
        pytest.skip("oracle/_ref/chkn-run not built")
    d = str(tmp_path / "ffs")
    shutil.copytree(FFS, d)
    import json
    with open(os.path.join(d, "config.json")) as f:
        cfg = json.load(f)
    cfg["max_step"] = 25
    with open(os.path.join(d, "config.json"), "w") as f:
        json.dump(cfg, f)
    # chicken's binary files (same values as the gzipped text): the flow is written back
    # at full precision (the text format keeps 6 significant digits)
    job = chicken.ChickenJob(d)
    for b in job.blocks:
        nic, njc, nkc = job.shape(b)
        name = f"{b[0]:04d}-{b[1]:04d}-{b[2]:04d}"
        verts = chicken.read_grid(os.path.join(d, "grid", f"grid-{name}.gz"), nic, njc, nkc)
        hdr = np.array([3.0, 0.0, 0.0, nic + 1, njc + 1, nkc + 1])
        with open(os.path.join(d, "grid", f"grid-{name}.bin"), "wb") as f:
            f.write(hdr.tobytes() + np.ascontiguousarray(verts.reshape(-1, 3)).tobytes())
        fl = chicken.read_flow(os.path.join(d, "flow", "t0000", f"flow-{name}.gz"), nic * njc * nkc, job.iovars)
        np.concatenate([fl[v] for v in job.iovars]).tofile(os.path.join(d, "flow", "t0000", f"flow-{name}.bin"))
    r = subprocess.run([cj.EXE, "--job=ffs", "--binary"], capture_output=True, text=True, cwd=str(tmp_path))
    assert r.returncode == 0, r.stdout[-400:] + r.stderr[-400:]
    tdirs = sorted(x for x in os.listdir(os.path.join(d, "flow")) if x.startswith("t"))
    s, job, index, _ = oracle_from_job(FFS, chicken_mode=True)
    assert s.run(25) == 0
    for b, n in index.items():
        nic, njc, nkc = job.shape(b)
        fc = chicken.read_flow(os.path.join(d, "flow", tdirs[-1], f"flow-{b[0]:04d}-{b[1]:04d}-{b[2]:04d}.bin"),
                               nic * njc * nkc, job.iovars)
        fo = s.get_flow(n)
        speed = np.max(np.hypot(fc["velx"], fc["vely"]))
        for key, ck in (("rho", "rho"), ("vx", "velx"), ("vy", "vely"), ("p", "p"), ("T", "T")):
            # velocity components against the speed (chicken's vertex-derived face normals
            # leave ~1e-13 m/s in the components that are zero on the exact grid)
            scale = speed if key in ("vx", "vy") else np.max(np.abs(fc[ck]))
            assert np.max(np.abs(fo[key] - fc[ck])) <= 1e-12 * scale, (b, key)


@pytest.mark.gpu
def test_ffs_job_on_gpu_matches_oracle():
    """The reference's forward-facing-step job dir loaded unchanged by gdfv.chicken (21
    active blocks, 4 inactive; inflow, exchange, outflow and default slip-wall tags) and
    run in FP64 on the GPU: per-cell agreement with the oracle set up from the same
    directory (Eilmer-4 options) to 1e-12 after 40 steps; then on to t = 1 ms, where the
    GPU path's shock (Eilmer's predictor-corrector, clipping and entropy fix) stands
    within one cell of the position chicken's scheme gives."""
    sim, job = chicken.load_job(FFS)
    s, _, index, geom = oracle_from_job(FFS, chicken_mode=False)
    assert set(index) == set(job.index)
    for b, n in index.items():   # the same conserved start on both sides
        sim.set_conserved(job.index[b], s.get_U(n))
        assert s.set_U(n, s.get_U(n)) == 0
    assert s.run(40) == 0
    assert sim.run(max_step=40) == 40
    for b, n in index.items():
        errs = cases.cell_errors(sim.get_conserved(job.index[b]), s.get_U(n), False)
        assert max(errs.values()) <= 1e-12, (b, errs)
    sim.run(max_step=job.cfg["max_step"], max_time=job.cfg["max_time"])
    nic, njc, nkc = job.shape((0, 0, 0))
    p = sim.get_flow(job.index[(0, 0, 0)])["p"].reshape(nkc, njc, nic)[0, 0, :]
    (dx, _, _), (x0, _, _) = geom[(0, 0, 0)]
    xn, cell = shock_position(p, x0 + (np.arange(nic) + 0.5) * dx)
    assert abs(xn - FFS_SHOCK_X) < cell, (xn, FFS_SHOCK_X)


@pytest.mark.gpu
def test_ffs_job_float_flux_matches_oracle():
    """The same job in the float-flux form: blocks two cells deep with slip walls on both
    k faces (the stencil planes beyond them are mirrored ghosts), inactive neighbours and
    default walls; relative L2 of rho, momentum and energy against the FP64 oracle
    <= 1e-6 after 40 steps."""
    sim, job = chicken.load_job(FFS, flux_precision="fp32")
    s, _, index, _ = oracle_from_job(FFS, chicken_mode=False)
    for b, n in index.items():
        sim.set_conserved(job.index[b], s.get_U(n))
        assert s.set_U(n, s.get_U(n)) == 0
    assert s.run(40) == 0
    assert sim.run(max_step=40) == 40
    Ug = np.concatenate([sim.get_conserved(job.index[b]) for b in index], axis=1)
    Uo = np.concatenate([s.get_U(n) for n in index.values()], axis=1)
    errs = [cases.rel_l2(Ug[0], Uo[0]), cases.rel_l2(Ug[1:4].ravel(), Uo[1:4].ravel()), cases.rel_l2(Ug[4], Uo[4])]
    assert max(errs) <= 1e-6, errs
