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
