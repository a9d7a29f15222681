"""Run a chicken job directory on the GPU path, and write its flow files back.

chicken (the reference's structured-grid CUDA solver) keeps a job as a directory:
  config.json                  the prep output read by src/chicken/config.cu:347-525
                               (read_config_file): lattice nib x njb x nkb, per-axis
                               cell counts nics/njcs/nkcs, blk_ids, fluid_blocks with
                               their face tags, flow_states, gas_model, x_order,
                               flux_calc, dt_init, max_time, max_step, cfl_values
  grid/grid-IIII-JJJJ-KKKK.bin|.gz   vertices (src/chicken/block.cu:786-879 readGrid)
  flow/tNNNN/flow-IIII-JJJJ-KKKK.bin|.gz   one IO variable after another, cells i
                               fastest (block.cu:882-975 readFlow / writeFlow, IO
                               variable order from config "iovar_names", cell.cu:66-68)
  times.data                   "tindx time" lines (simulate.cu:133-147, :176-177)

`load_job` builds a `Simulation` from such a directory: each block becomes a
uniform Cartesian block, or a graded rectilinear one where the spacing varies along
an axis (the grid must be axis-aligned), the face tags map onto this library's boundary conditions
(exchange -> full-face exchange with the lattice neighbour, wrapping periodically
at the lattice edge as chicken's index wrap does (face.cu:22-36); inflow -> supersonic
inflow of the tagged flow state; outflow -> extrapolation, xOrder 0; wall_with_slip
-> slip wall), and the cells start from the flow file's rho, T and velocity.
`write_flow` writes the state back in chicken's format and appends times.data.

The GPU path computes with Eilmer's options (predictor-corrector, face-frame l2r2
with extrema clipping and the AUSMDV entropy fix): a chicken job run here is that
scheme on chicken's grid, boundary tags and initial state, not chicken's own TVD-RK3
variant.  chicken's wall_no_slip_* and inflow_function tags are not on this path
and raise ValueError.
"""
import gzip
import json
import os

import numpy as np

from .solver import (Config, ExchangeBC_FullFace, FlowState, IdealGas, InFlowBC_Supersonic,
                     OutFlowBC_SimpleExtrapolate, Simulation, WallBC_WithSlip)

FACES = ("iminus", "iplus", "jminus", "jplus", "kminus", "kplus")
_FACE_NAME = {"iminus": "west", "iplus": "east", "jminus": "south", "jplus": "north",
              "kminus": "bottom", "kplus": "top"}
_OPPOSITE = {"iminus": "iplus", "iplus": "iminus", "jminus": "jplus", "jplus": "jminus",
             "kminus": "kplus", "kplus": "kminus"}
DEFAULT_IOVARS = ["posx", "posy", "posz", "vol", "p", "T", "rho", "e", "YB", "a", "velx", "vely", "velz"]


def _name(prefix, i, j, k, binary):
    return f"{prefix}-{i:04d}-{j:04d}-{k:04d}" + (".bin" if binary else ".gz")


def read_grid(path, nic, njc, nkc):
    """Vertices (nkv, njv, niv, 3) of a chicken grid file, binary or gzipped text."""
    niv, njv, nkv = nic + 1, njc + 1, nkc + 1
    if path.endswith(".bin"):
        raw = np.fromfile(path, dtype=np.float64)
        dims = [int(raw[3]), int(raw[4]), int(raw[5])]
        xyz = raw[6:]
    else:
        with gzip.open(path, "rt") as f:
            lines = f.read().splitlines()
        dims = [int(lines[3].split(":")[1]), int(lines[4].split(":")[1]), int(lines[5].split(":")[1])]
        xyz = np.array([float(v) for ln in lines[6:] if ln.strip() for v in ln.split()[:3]])
    if dims != [niv, njv, nkv]:
        raise ValueError(f"{path}: grid of {dims} vertices, expected {[niv, njv, nkv]}")
    return xyz.reshape(nkv, njv, niv, 3)


def uniform_geometry(verts, path=""):
    """(dx, dy, dz) and origin of an axis-aligned grid with constant spacing."""
    x, y, z = verts[0, 0, :, 0], verts[0, :, 0, 1], verts[:, 0, 0, 2]
    d = []
    for axis, line in enumerate((x, y, z)):
        steps = np.diff(line)
        if len(steps) == 0 or not np.all(steps > 0) or np.ptp(steps) > 1e-9 * steps.mean():
            raise ValueError(f"{path}: spacing along axis {axis} is not uniform")
        d.append(float(steps.mean()))
    expect = (verts[0, 0, 0][None, None, None, :] +
              np.stack(np.meshgrid(np.arange(verts.shape[0]) * d[2], np.arange(verts.shape[1]) * d[1],
                                   np.arange(verts.shape[2]) * d[0], indexing="ij")[::-1], axis=-1))
    if np.max(np.abs(verts - expect)) > 1e-9 * max(d) * max(verts.shape):
        raise ValueError(f"{path}: grid is not an axis-aligned Cartesian block")
    return tuple(d), tuple(float(v) for v in verts[0, 0, 0])


def rectilinear_vertices(verts, path=""):
    """(xv, yv, zv) of an axis-aligned grid whose spacing may vary along each axis (each
    vertex coordinate depends on its own index only)."""
    xv, yv, zv = verts[0, 0, :, 0], verts[0, :, 0, 1], verts[:, 0, 0, 2]
    for axis, line in enumerate((xv, yv, zv)):
        if not np.all(np.diff(line) > 0):
            raise ValueError(f"{path}: vertex coordinates along axis {axis} do not increase")
    Z, Y, X = np.meshgrid(zv, yv, xv, indexing="ij")
    expect = np.stack([X, Y, Z], axis=-1)
    scale = max(np.ptp(xv), np.ptp(yv), np.ptp(zv))
    if np.max(np.abs(verts - expect)) > 1e-12 * scale:
        raise ValueError(f"{path}: grid is not an axis-aligned rectilinear block")
    return xv.copy(), yv.copy(), zv.copy()


def read_flow(path, ncells, iovars):
    """dict IO-variable name -> values (ncells, i fastest) of a chicken flow file."""
    if path.endswith(".bin"):
        raw = np.fromfile(path, dtype=np.float64)
    else:
        with gzip.open(path, "rt") as f:
            raw = np.array([float(v) for v in f.read().split()])
    if raw.size != len(iovars) * ncells:
        raise ValueError(f"{path}: {raw.size} values, expected {len(iovars)} x {ncells}")
    raw = raw.reshape(len(iovars), ncells)
    return {name: raw[m] for m, name in enumerate(iovars)}


class ChickenJob:
    """The parts of a chicken job directory the GPU path uses (no GPU needed)."""

    def __init__(self, jobdir, tindx=0):
        self.jobdir = jobdir
        with open(os.path.join(jobdir, "config.json")) as f:
            self.cfg = cfg = json.load(f)
        self.nib, self.njb, self.nkb = cfg["nib"], cfg["njb"], cfg["nkb"]
        self.nics, self.njcs, self.nkcs = cfg["nics"], cfg["njcs"], cfg["nkcs"]
        self.iovars = cfg.get("iovar_names", DEFAULT_IOVARS)
        gm = cfg.get("gas_model", {})
        self.gamma = float(gm.get("gamma", 1.4))
        self.R = float(gm.get("R", 287.1))
        self.flow_states = [dict(p=fs["gas"]["p"], T=fs["gas"]["T"], vel=list(fs["vel"])) for fs in cfg["flow_states"]]
        self.blocks = {}   # (i, j, k) -> dict(bcs, active)
        for fb in cfg["fluid_blocks"]:
            self.blocks[(fb["i"], fb["j"], fb["k"])] = dict(bcs=fb["bcs"], active=fb.get("active", True))
        self.tindx = tindx
        self.time = self._start_time(tindx)
        self.binary = os.path.exists(os.path.join(jobdir, "grid", _name("grid", 0, 0, 0, True)))

    def _start_time(self, tindx):
        path = os.path.join(self.jobdir, "times.data")
        t = 0.0
        if os.path.exists(path):
            with open(path) as f:
                for line in f:
                    if not line.strip() or "#" in line:
                        continue
                    parts = line.split()
                    if int(parts[0]) == tindx:
                        t = float(parts[1])
        return t

    def active_blocks(self):
        return [b for b in sorted(self.blocks, key=lambda b: (b[2], b[1], b[0])) if self.blocks[b]["active"]]

    def shape(self, b):
        return self.nics[b[0]], self.njcs[b[1]], self.nkcs[b[2]]

    def neighbour(self, b, face):
        """Lattice neighbour across an exchange face (periodic wrap at the edges)."""
        axis = FACES.index(face) // 2
        step = 1 if face.endswith("plus") else -1
        n = [self.nib, self.njb, self.nkb]
        o = list(b)
        o[axis] = (o[axis] + step) % n[axis]
        return tuple(o)

    def solver_config(self, **overrides):
        cfg = self.cfg
        if cfg.get("x_order", 2) != 2:
            raise ValueError("only x_order 2 (l2r2 reconstruction) is on this path")
        flux = cfg.get("flux_calc", "ausmdv")
        if flux != "ausmdv":
            raise ValueError(f"flux_calc {flux!r} is not on this path")
        cfl = cfg.get("cfl_values", [0.5])
        kw = dict(flux_calculator="ausmdv", cfl_value=float(cfl[0]), dt_init=float(cfg.get("dt_init", 1.0e-6)),
                  dt_max=float(cfg.get("dt_max", 1.0e-3)), cfl_count=int(cfg.get("cfl_count", 10)))
        kw.update(overrides)
        return Config(**kw)


def load_job(jobdir, tindx=0, **config_overrides):
    """Build and prepare a Simulation from a chicken job directory; the state starts
    from flow/tNNNN (tindx) and the clock from times.data.  Returns (sim, job)."""
    job = ChickenJob(jobdir, tindx)
    sim = Simulation(job.solver_config(**config_overrides), gas=IdealGas(R=job.R, gamma=job.gamma))
    index = {}
    geom = {}
    for b in job.active_blocks():
        nic, njc, nkc = job.shape(b)
        path = os.path.join(jobdir, "grid", _name("grid", *b, job.binary))
        verts = read_grid(path, nic, njc, nkc)
        try:
            d, origin = uniform_geometry(verts, path)
            geom[b] = (d, origin)
            index[b] = sim.add_block(nic, njc, nkc, *d, *origin)
        except ValueError:   # stretched spacing: a graded rectilinear block
            xv, yv, zv = rectilinear_vertices(verts, path)
            geom[b] = (xv, yv, zv)
            index[b] = sim.add_block_graded(xv, yv, zv)
    for b in job.active_blocks():
        for face in FACES:
            bc = job.blocks[b]["bcs"].get(face, {"tag": "wall_with_slip"})
            tag = bc["tag"]
            if tag == "exchange":
                o = job.neighbour(b, face)
                if o not in index:
                    raise ValueError(f"block {b} exchanges across {face} with inactive block {o}")
                spec = ExchangeBC_FullFace(index[o], _FACE_NAME[_OPPOSITE[face]])
            elif tag == "inflow":
                fs = job.flow_states[bc["flow_state_index"]]
                spec = InFlowBC_Supersonic(FlowState(p=fs["p"], T=fs["T"], velx=fs["vel"][0], vely=fs["vel"][1],
                                                     velz=fs["vel"][2]))
            elif tag == "outflow":
                spec = OutFlowBC_SimpleExtrapolate(xOrder=0)
            elif tag == "wall_with_slip":
                spec = WallBC_WithSlip()
            else:
                raise ValueError(f"chicken boundary tag {tag!r} is not on this path")
            sim.set_bc(index[b], _FACE_NAME[face], spec)
    sim.prepare()
    for b in job.active_blocks():
        nic, njc, nkc = job.shape(b)
        path = os.path.join(jobdir, "flow", f"t{tindx:04d}", _name("flow", *b, job.binary))
        fl = read_flow(path, nic * njc * nkc, job.iovars)
        shp = (nkc, njc, nic)
        sim.set_flow_rhoT(index[b], fl["rho"].reshape(shp),
                          tuple(fl[v].reshape(shp) for v in ("velx", "vely", "velz")), fl["T"].reshape(shp))
    if job.time:
        t = sim.time()
        sim.set_time(job.time, 0, t["dt"])
    job.index = index
    job.geom = geom
    return sim, job


def write_flow(sim, job, tindx, time=None):
    """Write the current state as flow/tNNNN in chicken's format (binary or gzipped
    text as the job's grid files are) and append "tindx time" to times.data."""
    outdir = os.path.join(job.jobdir, "flow", f"t{tindx:04d}")
    os.makedirs(outdir, exist_ok=True)
    g, R = job.gamma, job.R
    cv = R / (g - 1.0)
    for b in job.active_blocks():
        nic, njc, nkc = job.shape(b)
        gb = job.geom[b]
        if len(gb) == 3:   # graded: vertex coordinates per axis
            cx, cy, cz = (0.5 * (v[1:] + v[:-1]) for v in gb)
            vol = np.einsum("k,j,i->kji", np.diff(gb[2]), np.diff(gb[1]), np.diff(gb[0])).ravel()
        else:
            (dx, dy, dz), (x0, y0, z0) = gb
            cx, cy, cz = (o + h * (np.arange(m) + 0.5) for o, h, m in ((x0, dx, nic), (y0, dy, njc), (z0, dz, nkc)))
            vol = np.full(nic * njc * nkc, dx * dy * dz)
        U = sim.get_conserved(job.index[b])
        rho = U[0]
        vel = U[1:4] / rho
        e = U[4] / rho - 0.5 * np.sum(vel * vel, axis=0)
        T = e / cv
        p = rho * R * T
        zc, yc, xc = np.meshgrid(cz, cy, cx, indexing="ij")
        n = nic * njc * nkc
        values = dict(posx=xc.ravel(), posy=yc.ravel(), posz=zc.ravel(), vol=vol, p=p, T=T,
                      rho=rho, e=e, YB=np.zeros(n), a=np.sqrt(g * R * T), velx=vel[0], vely=vel[1], velz=vel[2])
        data = np.concatenate([np.asarray(values[v], dtype=np.float64).ravel() for v in job.iovars])
        path = os.path.join(outdir, _name("flow", *b, job.binary))
        if job.binary:
            data.tofile(path)
        else:
            with gzip.open(path, "wt") as f:
                f.write("\n".join(repr(float(v)) for v in data) + "\n")
    t = sim.time()["time"] if time is None else time
    with open(os.path.join(job.jobdir, "times.data"), "a") as f:
        f.write(f"{tindx} {t}\n")


def main(argv=None):
    """python -m gdfv.chicken JOBDIR [--tindx N] [--steps N] [--precision fp64|fp32]:
    run a chicken job on the GPU path from flow/tNNNN for the config's max_step (or
    --steps) steps up to its max_time, and write the result as the next flow index."""
    import argparse
    ap = argparse.ArgumentParser(prog="python -m gdfv.chicken")
    ap.add_argument("jobdir")
    ap.add_argument("--tindx", type=int, default=0)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    args = ap.parse_args(argv)
    sim, job = load_job(args.jobdir, args.tindx, flux_precision=args.precision)
    steps = args.steps if args.steps is not None else int(job.cfg.get("max_step", 100))
    taken = sim.run(max_step=steps, max_time=float(job.cfg.get("max_time", 0.0)))
    write_flow(sim, job, args.tindx + 1)
    t = sim.time()
    print(f"{taken} steps to t = {t['time']:.6e} s (dt {t['dt']:.3e}); flow written as t{args.tindx + 1:04d}")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
