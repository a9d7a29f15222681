"""Regenerate the golden fixtures in tests/golden/ (run from the repository root).

chicken_lattice.npz -- final flow of a small two-block job run by the reference's
    own compiled chicken CPU solver (oracle/_ref/chkn-run, built from the read-only
    reference tree by `make -C oracle chicken`): 2 x (8 x 4 x 4) cells, M=3 inflow /
    exchange / outflow / slip walls, seeded 1% density noise, AUSMDV x_order 2,
    TVD-RK3, fixed dt = 2e-7 s, 12 steps.
reference_job_answers.json -- the numbers the reference's own integration tests
    assert (transcribed with their source lines; no run needed).
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def chicken_lattice_job():
    import chicken_job as cj
    d = 1.0 / 1024
    job = cj.LatticeJob([8, 8], [4], [4], d)
    T = 220.0
    u = 3 * np.sqrt(cj.GAMMA * cj.R * T)
    job.inflow = (5e3, T, (u, 0.0, 0.0))
    rng = np.random.default_rng(11)
    rho_inf = 5e3 / (cj.R * T)
    for b in job.blocks():
        job.flow[b] = (rho_inf * (1 + 0.01 * rng.standard_normal((4, 4, 8))), (u, 0.0, 0.0), T)
    job.bcs[((0, 0, 0), "iminus")] = "inflow"
    job.bcs[((1, 0, 0), "iplus")] = "outflow"
    job.bcs[((0, 0, 0), "iplus")] = "exchange"
    job.bcs[((1, 0, 0), "iminus")] = "exchange"
    return job


DT, NSTEPS = 2.0e-7, 12

if __name__ == "__main__":
    import chicken_job as cj
    job = chicken_lattice_job()
    flow, _, _ = cj.run(job, DT, NSTEPS)
    out = {}
    for b, f in flow.items():
        for k, v in f.items():
            out[f"b{b[0]}{b[1]}{b[2]}_{k}"] = v
    for b in job.blocks():
        rho, vel, T = job.flow[b]
        out[f"init_b{b[0]}{b[1]}{b[2]}_rho"] = np.asarray(rho)
    np.savez_compressed(os.path.join(HERE, "chicken_lattice.npz"), **out)
    answers = {
        "sod": {"source": "examples/eilmer/3D/sod-shock-tube/sg/sod-test.rb:32-90",
                "steps": 75, "steps_tol": 3, "max_time": 0.6e-3,
                "probe_078": {"rho": 0.2647, "p": 30.2e3, "T": 398.0, "velx": 293.0},
                "probe_060": {"rho": 0.4271, "p": 30.2e3, "T": 247.0, "velx": 293.0}, "rel_tol": 1e-2},
        "mhd_shock_tube": {"source": "examples/eilmer/2D/MHDShockTube/MHD-ShockTube-Test.rb:36-80",
                           "steps": 880, "steps_tol": 10, "max_time": 6e-2,
                           "p": [1.84083e2, 1.84083e2, 1.84083e2], "vel.y": [-2.36600e-1, 0.0, 2.36599e-1],
                           "vel.z": [-5.71203e-1, 0.0, -5.71203e-1], "B.y": [4.00346, 5.66174, 4.00346],
                           "B.z": [-4.00346, -1.23741e-7, 4.00346], "rho": [3.90913, 3.90913, 3.90913],
                           "tol": {"p": 1e1, "vel.y": 1e-2, "vel.z": 1e-2, "B.y": 1e-1, "B.z": 1e-1, "rho": 1e-1}},
    }
    with open(os.path.join(HERE, "reference_job_answers.json"), "w") as f:
        json.dump(answers, f, indent=1)
    print("wrote golden fixtures")
