"""Run the reference's own compiled chicken CPU solver (oracle/_ref/chkn-run) on a
job written here, and read its flow files back.

TEST INFRASTRUCTURE ONLY: used to pin the CPU oracle against real reference code
(tests/test_chicken_pin.py) and, in bench.py's reference arm, to time the
reference's CPU path.  The job files follow chicken's formats:
  config.json        src/chicken/config.cu:347-525 (read_config_file)
  grid/*.bin         src/chicken/block.cu:786-828 (readGrid, binary)
  flow/tNNNN/*.bin   src/chicken/block.cu:882-907 (readFlow, binary, IOvar order
                     of src/chicken/cell.cu:66-68)
Chicken's only gas model here is its compiled-in ideal air (gamma 1.4, R 287.1,
src/chicken/gas.cu:33-40) and its only time scheme TVD-RK3.
"""
import glob
import json
import os
import shutil
import subprocess
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
EXE = os.path.join(HERE, "_ref", "chkn-run")
GAMMA, R = 1.4, 287.1
CV = R / (GAMMA - 1.0)
IOVARS = ["posx", "posy", "posz", "vol", "p", "T", "rho", "e", "YB", "a", "velx", "vely", "velz"]
FACES = ["iminus", "iplus", "jminus", "jplus", "kminus", "kplus"]


def available():
    return os.path.exists(EXE)


class LatticeJob:
    """A chicken job: nib x njb x nkb blocks with per-axis cell counts, uniform spacing d.
    bcs maps (block (i,j,k), face name) -> tag; unspecified faces are slip walls.
    Initial state per block from rho, vel (3 arrays), T, each shaped (nkc, njc, nic)."""

    def __init__(self, nics, njcs, nkcs, d):
        self.nics, self.njcs, self.nkcs = list(nics), list(njcs), list(nkcs)
        self.d = float(d)
        self.nib, self.njb, self.nkb = len(nics), len(njcs), len(nkcs)
        self.bcs = {}
        self.inflow = None
        self.flow = {}

    def blocks(self):
        for k in range(self.nkb):
            for j in range(self.njb):
                for i in range(self.nib):
                    yield (i, j, k)

    def blk_id(self, i, j, k):
        return i + self.nib * (j + self.njb * k)

    def origin(self, i, j, k):
        return (self.d * sum(self.nics[:i]), self.d * sum(self.njcs[:j]), self.d * sum(self.nkcs[:k]))

    def write(self, jobdir, dt, nsteps):
        os.makedirs(os.path.join(jobdir, "grid"), exist_ok=True)
        os.makedirs(os.path.join(jobdir, "flow", "t0000"), exist_ok=True)
        blk_ids = [[[0] * self.nkb for _ in range(self.njb)] for _ in range(self.nib)]
        fluid_blocks = []
        for (i, j, k) in self.blocks():
            bid = self.blk_id(i, j, k)
            blk_ids[i][j][k] = bid
            bcs = {}
            for f in FACES:
                tag = self.bcs.get(((i, j, k), f), "wall_with_slip")
                entry = {"tag": tag}
                if tag == "inflow":
                    entry["flow_state_index"] = 0
                bcs[f] = entry
            fluid_blocks.append({"i": i, "j": j, "k": k, "active": True, "bcs": bcs})
        flow_states = []
        if self.inflow is not None:
            p, T, vel = self.inflow
            flow_states.append({"gas": {"p": p, "T": T, "YB": 0.0}, "vel": list(vel)})
        else:
            flow_states.append({"gas": {"p": 1.0e5, "T": 300.0, "YB": 0.0}, "vel": [0.0, 0.0, 0.0]})
        cfg = {
            "title": "gdfv pin", "gas_model": {"gamma": GAMMA, "R": R, "q": 0.0, "alpha": 0.0, "Ti": 0.0, "Cv": CV},
            "iovar_names": IOVARS, "n_flow_states": len(flow_states), "flow_states": flow_states,
            "n_fluid_blocks": self.nib * self.njb * self.nkb, "nib": self.nib, "njb": self.njb, "nkb": self.nkb,
            "nics": self.nics, "njcs": self.njcs, "nkcs": self.nkcs, "blk_ids": blk_ids,
            "fluid_blocks": fluid_blocks, "x_order": 2, "t_order": 3, "flux_calc": "ausmdv",
            "source_terms": "none", "dt_init": dt, "max_time": 1.0e9, "max_step": nsteps,
            "cfl_times": [0.0], "cfl_values": [0.5], "cfl_count": nsteps + 10, "print_count": nsteps + 10,
            "t_change": [0.0], "dt_plot": [1.0e9], "reacting": False, "viscous": False,
            "threads_per_gpu_block": 128,
        }
        with open(os.path.join(jobdir, "config.json"), "w") as f:
            json.dump(cfg, f)
        for (i, j, k) in self.blocks():
            nic, njc, nkc = self.nics[i], self.njcs[j], self.nkcs[k]
            x0, y0, z0 = self.origin(i, j, k)
            xs = x0 + self.d * np.arange(nic + 1)
            ys = y0 + self.d * np.arange(njc + 1)
            zs = z0 + self.d * np.arange(nkc + 1)
            Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
            verts = np.stack([X, Y, Z], axis=-1).reshape(-1, 3)
            hdr = np.array([3.0, 0.0, 0.0, nic + 1, njc + 1, nkc + 1], dtype=np.float64)
            with open(os.path.join(jobdir, "grid", f"grid-{i:04d}-{j:04d}-{k:04d}.bin"), "wb") as f:
                f.write(hdr.tobytes())
                f.write(np.ascontiguousarray(verts, dtype=np.float64).tobytes())
            rho, vel, T = self.flow[(i, j, k)]
            shp = (nkc, njc, nic)
            rho = np.broadcast_to(rho, shp).astype(np.float64)
            T = np.broadcast_to(T, shp).astype(np.float64)
            vx, vy, vz = (np.broadcast_to(v, shp).astype(np.float64) for v in vel)
            # GasState.update_from_pT consistency: p = rho R T, e = Cv T, a = sqrt(g R T)
            p = rho * R * T
            e = T * CV
            a = np.sqrt(GAMMA * R * T)
            zc, yc, xc = np.meshgrid(z0 + self.d * (np.arange(nkc) + 0.5), y0 + self.d * (np.arange(njc) + 0.5),
                                     x0 + self.d * (np.arange(nic) + 0.5), indexing="ij")
            vol = np.full(shp, self.d ** 3)
            data = [xc, yc, zc, vol, p, T, rho, e, np.zeros(shp), a, vx, vy, vz]
            with open(os.path.join(jobdir, "flow", "t0000", f"flow-{i:04d}-{j:04d}-{k:04d}.bin"), "wb") as f:
                for arr in data:
                    f.write(np.ascontiguousarray(arr, dtype=np.float64).ravel().tobytes())

    def read(self, jobdir):
        """Final flow of every block: dict (i,j,k) -> {iovar: array (nkc*njc*nic)}."""
        tdirs = sorted(glob.glob(os.path.join(jobdir, "flow", "t*")))
        last = tdirs[-1]
        out = {}
        for (i, j, k) in self.blocks():
            n = self.nics[i] * self.njcs[j] * self.nkcs[k]
            raw = np.fromfile(os.path.join(last, f"flow-{i:04d}-{j:04d}-{k:04d}.bin"), dtype=np.float64)
            raw = raw.reshape(len(IOVARS), n)
            out[(i, j, k)] = {name: raw[m] for m, name in enumerate(IOVARS)}
        return out


def run(job, dt, nsteps, threads=None, keep=None, exe=EXE):
    """Write, run and read a job; returns (flow dict, wall seconds of the solver run)."""
    jobdir = keep or tempfile.mkdtemp(prefix="chkn_")
    try:
        job.write(jobdir, dt, nsteps)
        env = dict(os.environ)
        if threads:
            env["OMP_NUM_THREADS"] = str(threads)
        t0 = time.perf_counter()
        r = subprocess.run([os.path.abspath(exe), f"--job={jobdir}", "--binary"], capture_output=True, text=True, env=env,
                           cwd=os.path.dirname(jobdir) or ".")
        wall = time.perf_counter() - t0
        if r.returncode != 0 or "bad cell" in r.stdout.lower() + r.stderr.lower():
            raise RuntimeError(f"chkn-run failed: {r.stdout[-500:]} {r.stderr[-500:]}")
        return job.read(jobdir), wall, r.stdout
    finally:
        if keep is None:
            shutil.rmtree(jobdir, ignore_errors=True)


def march_seconds(stdout):
    """Seconds chicken spent after its start-up, from its own printout (None if absent)."""
    import re
    done = re.search(r"Done in ([0-9.eE+-]+)\s*s", stdout)
    init = re.search(r"initialize_simulation\(\) finished in ([0-9.eE+-]+)\s*ms", stdout)
    if not done or not init:
        return None
    return float(done.group(1)) - 1e-3 * float(init.group(1))


def bench(exe=EXE, steps=10, warmup=3, n=96, nblk=(4, 4, 4), seed=4321):
    """Reference-arm timing: chicken (OpenMP over blocks) on an n^3 sample of the M=3
    inflow box split into nblk blocks so that every host core has a block (the
    threads that can work, min(cores, blocks), are reported as `cores`)."""
    cores = len(os.sched_getaffinity(0))
    nb = nblk
    job = LatticeJob([n // nb[0]] * nb[0], [n // nb[1]] * nb[1], [n // nb[2]] * nb[2], 1.0 / 1024)
    T = 220.0
    u = 3.0 * np.sqrt(GAMMA * R * T)
    job.inflow = (5.0e3, T, (u, 0.0, 0.0))
    rng = np.random.default_rng(seed)
    rho_inf = 5.0e3 / (R * T)
    for (i, j, k) in job.blocks():
        shp = (job.nkcs[k], job.njcs[j], job.nics[i])
        job.flow[(i, j, k)] = (rho_inf * (1 + 0.01 * rng.standard_normal(shp)), (u, 0.0, 0.0), T)
        if i == 0:
            job.bcs[((i, j, k), "iminus")] = "inflow"
        if i == nb[0] - 1:
            job.bcs[((i, j, k), "iplus")] = "outflow"
        for f, cond in (("iminus", i > 0), ("iplus", i < nb[0] - 1), ("jminus", j > 0), ("jplus", j < nb[1] - 1),
                        ("kminus", k > 0), ("kplus", k < nb[2] - 1)):
            if cond:
                job.bcs[((i, j, k), f)] = "exchange"
    dt = 0.5 * (1.0 / 1024) / (u + np.sqrt(GAMMA * R * T)) / 2
    # per-step time from the difference of a short and a long run (start-up and
    # job I/O cancel); at least 10 timed steps so that the difference is resolved
    steps, warmup = max(int(steps), 10), max(int(warmup), 1)
    _, w_small, out_small = run(job, dt, warmup, threads=cores, exe=exe)
    _, w_big, out_big = run(job, dt, warmup + steps, threads=cores, exe=exe)
    # chicken's own clock of the time march: "Done in" (simulate.cu) less its start-up
    # ("initialize_simulation() finished in"); the flow write at the end cancels in the difference
    m_small, m_big = march_seconds(out_small), march_seconds(out_big)
    if m_small is not None and m_big is not None:
        w_small, w_big = m_small, m_big
    if w_big - w_small > 0.2 * w_big:
        per_step = (w_big - w_small) / steps
    else:   # difference not resolved: charge the whole long run to its steps
        per_step = w_big / (warmup + steps)
    value = n ** 3 / per_step / 1e6
    # chicken takes 3 stages per step (TVD-RK3) where the predictor-corrector takes 2
    return dict(value=value, cpu_baseline=dict(
        value=value, unit="Mcell-updates/s", cores=min(cores, nb[0] * nb[1] * nb[2]), kind="reference",
        sample=(f"reference chicken CPU build (oracle/_ref/chkn-run, OpenMP over blocks), {n}^3 cells of the "
                f"M=3 inflow box as {nb[0]}x{nb[1]}x{nb[2]} blocks, AUSMDV x_order 2, TVD-RK3 (3 stages/step), "
                f"{steps} timed steps (difference of a {warmup}- and a {warmup + steps}-step run)")))
