#!/usr/bin/env python
"""Benchmark of the explicit structured-grid FV update on B200.

Workload (one GPU): single block 256x256x256 ideal air (R=287.1, gamma=1.4), M=3
supersonic inflow (p=5e3 Pa, T=220 K) on x-min, extrapolate outflow on x-max, slip
walls on y/z, 1% seeded density noise, AUSMDV flux, l2r2 van Albada, predictor-
corrector.  A step is one full predictor-corrector step over all cells (with the
device-resident dt rule).  `value` is Mcell-updates/s of the FP32-flux / FP64-update
form; the plain FP64 form is timed beside it and both final states are compared
(relative L2 of rho, momentum, energy).

`--impl reference` times the reference's own CPU path: the compiled chicken solver
(oracle/_ref/chkn-run, TVD-RK3 AUSMDV, OpenMP over blocks) when it is present,
else the CPU oracle port (OpenMP over cells), on a bounded sample of the workload.

Multi-GPU (torchrun): every rank advances its own replica of the workload (the path
partitions into independent blocks; no collective on the data path), timed on the
device, max over ranks; value = all cells*steps / that time.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "gdtk-rmhd_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

METRIC = "Mcell-updates/s, FP32-flux vs FP64 plain at <=1e-6 rel L2 rho; adjoint/fwd time"
UNIT = "Mcell-updates/s"
BYTES_STAGE1 = 80    # read U0 (5 x 8 B), write dU0 (5 x 8 B) per cell
BYTES_STAGE2 = 120   # read U0 and dU0, write U2 per cell


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region: NVML polled every
    2 ms from a thread (nvidia-smi's loop, at 100 ms, when NVML is missing)."""

    REASONS = (("hw_slowdown", 0x8), ("sw_thermal_slowdown", 0x20), ("hw_thermal_slowdown", 0x40),
               ("sw_power_cap", 0x4))

    def __init__(self, index, interval=0.002):
        self.index = index
        self.interval = interval
        self.samples = []   # (sm_mhz, sm_max_mhz, reason bits)
        self.proc = None
        self._stop = threading.Event()
        self.thread = None

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            smax = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)

            def poll():
                while not self._stop.is_set():
                    try:
                        sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
                        bits = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                        self.samples.append((float(sm), float(smax), int(bits)))
                    except Exception:
                        pass
                    time.sleep(self.interval)

            self.thread = threading.Thread(target=poll, daemon=True)
            self.thread.start()
            return self
        except Exception:
            pass
        q = ("index,clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            f = [x.strip() for x in line.split(",")]
            try:
                bits = sum(b for (_, b), v in zip(self.REASONS, f[3:7]) if v.lower() == "active")
                self.samples.append((float(f[1]), float(f[2]), bits))
            except Exception:
                pass

    def __exit__(self, *a):
        self._stop.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=2)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [s[0] for s in self.samples]
        reasons = sorted({n for s in self.samples for n, b in self.REASONS if s[2] & b})
        return {"sm_mhz": float(np.median(sm)), "sm_min_mhz": float(min(sm)), "sm_max_mhz": max(s[1] for s in self.samples),
                "reasons": reasons, "samples": len(self.samples)}


def max_over_ranks(value, device="cpu"):
    """Max of a per-rank timing over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_oracle_baseline(cells_target=96, steps=24):
    """CPU oracle port (OpenMP over cells) on a bounded sample: 96^3 cells of the same workload."""
    import cases
    n = cells_target
    case = cases.c2_inflow_box(n=(n, n, n))
    orc = cases.build_oracle(case)
    orc.run(1)  # warm
    t0 = time.perf_counter()
    rc = orc.run(steps)
    dt = time.perf_counter() - t0
    cores = len(os.sched_getaffinity(0))
    return dict(value=n ** 3 * steps / dt / 1e6, unit=UNIT, cores=cores, kind="port",
                sample=f"CPU oracle (restatement of the Eilmer-4 path, OpenMP over cells), {n}^3 cells of the "
                       f"same M=3 inflow box, {steps} predictor-corrector steps, rc={rc}")


def chicken_baseline(steps, warmup):
    """The reference's chicken CPU build, if oracle/_ref holds it."""
    exe = os.path.join(ROOT, "oracle", "_ref", "chkn-run")
    if not os.path.exists(exe):
        return None
    try:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import chicken_job
    except Exception:
        return None
    return chicken_job.bench(exe, steps=steps, warmup=warmup)


def chicken_gpu_leg(n=128, steps=1000, warmup=20):
    """The reference's own GPU solver (chicken's CUDA build for sm_100a,
    oracle/_ref/chkn-run-gpu: FP64, AUSMDV x_order 2, TVD-RK3, one thread per cell and
    per face) on the same M=3 inflow box as one block, timed on this GPU: per-step time
    from the difference of a short and a long run (start-up and binary job I/O cancel).
    Reported per step and per stage (TVD-RK3 takes 3 stages a step, the
    predictor-corrector 2)."""
    exe = os.path.join(ROOT, "oracle", "_ref", "chkn-run-gpu")
    if not os.path.exists(exe):
        return {"unavailable": "oracle/_ref/chkn-run-gpu not built (make -C oracle chicken_gpu)"}
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import chicken_job
    r = chicken_job.bench(exe, steps=steps, warmup=warmup, n=n, nblk=(1, 1, 1))
    per_step = r["value"]
    return dict(value=per_step, unit=UNIT, value_per_stage=per_step * 3,
                workload=f"M=3 inflow box {n}^3 as one block, FP64, TVD-RK3 (3 stages per step)",
                how=r["cpu_baseline"]["sample"].replace("reference chicken CPU build (oracle/_ref/chkn-run, "
                                                        "OpenMP over blocks)", "reference chicken GPU build"))


def adjoint_over_forward(nsteps=50, shape=(128, 128, 64), autotune=True, forms=(("resident", None), ("checkpointed", 10))):
    """Adjoint configuration: 128x128x64 M=3 inflow box (FP64, ausmdv), J = pressure
    integral over the y-min wall after 50 steps, gradient w.r.t. U0 and the inflow
    state through the rollout.  Returns the ratio of the backward time to the forward
    time of the same 50 steps run by gdfv_run with the autotuned schedule (the forward
    the library runs by default), both with CUDA events on the device and both warm (a
    rollout of the same length and its backward run first, so that torch's caching
    allocator holds the trajectory buffers).  Two backward forms: the trajectory resident
    in device memory (rollout's default when it fits: 100 states, 4.2 GB here), which
    recomputes nothing, and a checkpoint every 10 steps with each segment recomputed.
    Also the time of the rollout's own forward, which keeps the trajectory (gdfv_run_record:
    the steps and their records on the device, one host round trip), between events around
    the call: the minimum and the maximum of two warm passes (host work between the events,
    such as Python allocating the trajectory's tensors, adds to it and varies)."""
    import torch
    import cases
    from gdfv.autograd import rollout
    from test_gpu_adjoint import wall_pressure
    case = cases.c2_inflow_box(n=shape)
    inf = cases.inflow_state_m3()
    sim = cases.build_gpu(case, autotune=autotune)
    stream = torch.cuda.Stream()
    sim.set_stream(stream.cuda_stream)
    U0 = torch.from_numpy(sim.get_conserved(0)).cuda()
    sim.run(max_step=2)
    sim.set_conserved(0, U0.cpu().numpy())
    sim.set_time(0.0, 0, sim.config.dt_init)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.run(max_step=nsteps)
    e1.record(stream)
    torch.cuda.synchronize()
    fwd_ms = e0.elapsed_time(e1)
    out = dict(forward_ms=fwd_ms, steps=nsteps, workload=f"M=3 inflow box {shape[0]}x{shape[1]}x{shape[2]} FP64",
               forward_schedule="autotuned" if autotune else "default tiles")
    for label, K in forms:
        theta = torch.tensor([inf["p"], inf["T"], inf["vel"][0]], dtype=torch.float64, requires_grad=True)
        fwd_reps = []
        for rep in range(3):   # the first pass warms the adjoint (scratch allocation, face tables)
            theta.grad = None
            U0r = U0.clone().requires_grad_(True)
            f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            f0.record(stream)
            with torch.cuda.stream(stream):
                UN = rollout(sim, U0r, theta, nsteps, K)
            f1.record(stream)
            with torch.cuda.stream(stream):
                J = wall_pressure(case, UN, case.R)
            torch.cuda.synchronize()
            b0, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            b0.record()
            J.backward()
            b1.record()
            torch.cuda.synchronize()
            if rep:
                fwd_reps.append(f0.elapsed_time(f1))
        adj_ms = b0.elapsed_time(b1)
        out[label] = dict(ratio=adj_ms / fwd_ms, adjoint_ms=adj_ms, checkpoint_every=K or nsteps,
                          rollout_forward_ms=min(fwd_reps), rollout_forward_ms_max=max(fwd_reps),
                          forward_recorded_on_device=bool(getattr(sim, "rollout_recorded", False)),
                          dJ_dp_inflow=float(theta.grad[0]),
                          grad_U0_norm=float(U0r.grad.norm()))
    first = out[forms[0][0]]
    out.update(ratio=first["ratio"], adjoint_ms=first["adjoint_ms"], checkpoint_every=first["checkpoint_every"])
    return out


def adjoint_mhd_leg(stream, nsteps=30, n=(256, 256, 4)):
    """MHD rollout adjoint: Orszag-Tang 256x256x4 (FP64, hlle with GLM cleaning), J = <W, U_N>
    with fixed random weights after 30 steps, the trajectory resident; the backward time
    (each step's c_h and psi damping formed from its start state, then the two MHD VJP
    products) over the autotuned forward gdfv_run of the same steps, both warm."""
    import numpy as np
    import torch
    import cases
    from gdfv.autograd import rollout
    case = cases.orszag_tang(n=n)
    sim = cases.build_gpu(case, autotune=True)
    sim.set_stream(stream.cuda_stream)
    U0 = torch.from_numpy(sim.get_conserved(0)).cuda()
    sim.run(max_step=2)
    W = torch.from_numpy(np.random.default_rng(3).standard_normal(tuple(U0.shape))).cuda()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    fwd = []
    for _ in range(2):
        sim.set_conserved(0, U0.cpu().numpy())
        sim.set_time(0.0, 0, sim.config.dt_init)
        torch.cuda.synchronize()
        e0.record(stream)
        sim.run(max_step=nsteps)
        e1.record(stream)
        torch.cuda.synchronize()
        fwd.append(e0.elapsed_time(e1))
    fwd_ms = min(fwd)
    adj = []
    for rep in range(3):   # the first pass allocates the adjoint's scratch
        theta = torch.tensor([1.0, 1.0, 0.0], dtype=torch.float64, requires_grad=True)
        U0r = U0.clone().requires_grad_(True)
        with torch.cuda.stream(stream):
            UN = rollout(sim, U0r, theta, nsteps, nsteps)
            J = (UN * W).sum()
        torch.cuda.synchronize()
        b0, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        b0.record()
        J.backward()
        b1.record()
        torch.cuda.synchronize()
        if rep:
            adj.append(b0.elapsed_time(b1))
    adj_ms = min(adj)
    sim.close()
    return dict(workload=f"Orszag-Tang {n[0]}x{n[1]}x{n[2]} FP64 hlle+GLM, {nsteps} steps, trajectory resident",
                forward_ms=fwd_ms, adjoint_ms=adj_ms, adjoint_ms_max=max(adj), ratio=adj_ms / fwd_ms,
                grad_U0_norm=float(U0r.grad.norm()))


def _timed_run(sim, stream, steps):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.run(max_step=steps)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def _l2_errors(Uf, Ud, mhd=False):
    import cases
    err = dict(rho=cases.rel_l2(Uf[0], Ud[0]), momentum=cases.rel_l2(Uf[1:4].ravel(), Ud[1:4].ravel()),
               energy=cases.rel_l2(Uf[4], Ud[4]))
    if mhd:
        err["B"] = cases.rel_l2(Uf[5:8].ravel(), Ud[5:8].ravel())
    return err


def accuracy_leg(sims, n, flux, total_steps, stream):
    """FP32-flux against plain FP64 on the M=3 inflow box after `total_steps` steps
    from the same seeded state (both forms run their own dt rule)."""
    import cases
    out = {}
    if sims is None:
        sims = {}
        for prec in ("fp32", "fp64"):
            case = cases.c2_inflow_box(n=(n, n, n), flux=flux, precision=prec, seed=4321)
            sim = cases.build_gpu(case)
            sim.set_stream(stream.cuda_stream)
            sims[prec] = sim
    for prec, sim in sims.items():
        done = sim.time()["step"]
        if total_steps > done:
            sim.run(max_step=total_steps - done)
    Uf, Ud = sims["fp32"].get_conserved(0), sims["fp64"].get_conserved(0)
    out["steps"] = total_steps
    out["flux_calculator"] = flux
    if flux == "hllc":   # both forms equal the oracle; the oracle's hllc has no reference-held check
        out["pinned"] = "unpinned by the reference: no reference run, test or job uses hllc"
    out["rel_l2_vs_fp64"] = _l2_errors(Uf, Ud)
    out["time_fp32"], out["time_fp64"] = sims["fp32"].time()["time"], sims["fp64"].time()["time"]
    return out


def multiblock_leg(stream, steps=20, seed=2024):
    """Batched multi-block configuration: 64 blocks on a 4x4x4 lattice with per-axis
    sizes drawn by seed from {16,32,48,64,96,128}, full-face exchange inside, the M=3
    inflow box's boundary conditions outside; FP32 flux; tiles and launch form chosen
    by the autotuner on the first run."""
    import cases
    case = cases.multiblock_lattice(nb=(4, 4, 4), sizes=(16, 32, 48, 64, 96, 128), seed=seed, precision="fp32")
    cells = sum(int(np.prod(b["n"])) for b in case.blocks)
    sim = cases.build_gpu(case, autotune=True)
    sim.set_stream(stream.cuda_stream)
    sim.run(max_step=3)
    ms = _timed_run(sim, stream, steps)
    out = dict(workload=f"64-block lattice (4x4x4, sizes by seed {seed} from 16..128), FP32 flux",
               cells=cells, steps=steps, value=cells * steps / (ms * 1e-3) / 1e6, unit=UNIT,
               tile_kchunk=sim.option("tile_kchunk"), persistent=bool(sim.option("persistent")),
               tile_width=sim.option("tile_width"),
               autotune_stage_ms=sim.option("autotune_stage_ms"))
    sim.close()
    return out


def _max_divB(U, n, d):
    """max |div B| by central differences of the cell-centred field (periodic)."""
    nic, njc, nkc = n
    Bx = U[5].reshape(nkc, njc, nic)
    By = U[6].reshape(nkc, njc, nic)
    div = (np.roll(Bx, -1, axis=2) - np.roll(Bx, 1, axis=2)) / (2 * d[0]) + \
          (np.roll(By, -1, axis=1) - np.roll(By, 1, axis=1)) / (2 * d[1])
    return float(np.abs(div).max())


def mhd_leg(stream, steps=2000, n=(512, 512, 4), dt=8.0e-5):
    """Ideal-MHD Orszag-Tang vortex (hlle + GLM divergence cleaning, periodic, gamma
    5/3, 1% seeded density noise): plain FP64 and FP32-flux forms at one fixed dt
    (so that both compare at the same times; 2000 x 8e-5 = 0.16), throughput over
    the last 100 steps, error of the float form and max |div B| of both; beside the float
    form's error, that of the FP64 form started from a density perturbed by float-epsilon
    noise (the flow's sensitivity, which bounds what any float form can reach)."""
    import cases
    out = dict(workload=f"Orszag-Tang {n[0]}x{n[1]}x{n[2]} hlle+GLM, fixed dt {dt}", steps=steps)
    states = {}
    cells = int(np.prod(n))
    for prec in ("fp64", "fp32"):
        case = cases.orszag_tang(n=n, precision=prec)
        sim = cases.build_gpu(case, fixed_time_step=True, dt_init=dt, dt_max=dt)
        sim.set_stream(stream.cuda_stream)
        sim.run(max_step=steps - 100)
        ms = _timed_run(sim, stream, 100)
        out[f"value_{prec}"] = cells * 100 / (ms * 1e-3) / 1e6
        states[prec] = sim.get_conserved(0)
        out[f"max_divB_{prec}"] = _max_divB(states[prec], n, case.blocks[0]["d"])
        out[f"time_{prec}"] = sim.time()["time"]
        sim.close()
    out["unit"] = UNIT
    out["rel_l2_vs_fp64"] = _l2_errors(states["fp32"], states["fp64"], mhd=True)
    # the flow's own sensitivity: the FP64 form from a density perturbed once by float-epsilon
    # noise (relative 6e-8), against the unperturbed FP64 run at the same time
    case = cases.orszag_tang(n=n, precision="fp64")
    sim = cases.build_gpu(case, fixed_time_step=True, dt_init=dt, dt_max=dt)
    sim.set_stream(stream.cuda_stream)
    U0 = sim.get_conserved(0)
    U0[0] *= 1.0 + 6.0e-8 * np.random.default_rng(3).standard_normal(U0[0].shape)
    sim.set_conserved(0, U0)
    sim.run(max_step=steps)
    out["fp64_perturbed_6e-8_rel_l2_vs_fp64"] = _l2_errors(sim.get_conserved(0), states["fp64"], mhd=True)
    sim.close()
    return out


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    res = chicken_baseline(args.steps, args.warmup)
    one_block = None
    if res is None:
        base = cpu_oracle_baseline()
        res = dict(value=base["value"], cpu_baseline=base)
    else:
        try:   # the same solver on one block: OpenMP over blocks leaves one core working
            import chicken_job
            one_block = chicken_job.bench(steps=10, warmup=2, n=64, nblk=(1, 1, 1))["cpu_baseline"]
        except Exception as e:
            one_block = {"error": str(e)}
    line = {
        "metric": METRIC, "value": res["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "higher_is_better": True, "impl": "reference",
        "cpu_baseline": res["cpu_baseline"],
        "e2e": {"value": res["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "config": {"workload": "M=3 inflow box 256^3 (bounded CPU sample)", "flux_calculator": "ausmdv"},
        "data": "synthetic",
    }
    if one_block is not None:
        line["one_block"] = one_block
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--flux", default="ausmdv", choices=["ausmdv", "hllc"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--autotune", type=int, default=1, choices=[0, 1],
                    help="1: the library's autotuner picks the tile k-chunk and launch form on the first "
                         "(warm-up) run of each timed simulation")
    ap.add_argument("--accuracy-steps", type=int, default=1000,
                    help="steps after which the FP32 form is compared with FP64 (0: at the timed steps)")
    ap.add_argument("--no-extra", action="store_true", help="skip the multi-block, MHD and adjoint legs")
    ap.add_argument("--profile-case", nargs="?", const="stage", default=None,
                    choices=["stage", "corrector", "narrow", "mhd", "adjoint", "adjoint_mhd", "norms"],
                    help="small case for ncu captures, then exit: stage = the 128^3 inflow box "
                         "(FP32 then FP64 form, warmup steps); corrector = the inflow box at 256x128x128, "
                         "FP32 form, with the 256^3 run's tile k-chunk; narrow = the inflow box at "
                         "240x128x128, FP32 form in 16-wide tiles (the tuner's choice at 240^3); mhd = "
                         "Orszag-Tang 512x512x4 (both forms, warmup steps); adjoint = 128x128x64 FP64 "
                         "rollout of 10 steps and its backward; adjoint_mhd = Orszag-Tang 256x256x4 FP64 "
                         "rollout of 10 steps (resident) and its backward; norms = the 256^3 box, FP32 form, "
                         "warmup steps then the residual norms twice")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)

    import torch
    import torch.distributed as dist

    import cases

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    n = 128 if args.profile_case and args.profile_case != "norms" else args.size
    shape = (n, n, n)
    stream = torch.cuda.Stream()  # a capturable (non-default) stream shared with the library

    def make(prec):
        case = cases.c2_inflow_box(n=shape, flux=args.flux, precision=prec, seed=4321)
        sim = cases.build_gpu(case, autotune=bool(args.autotune))
        sim.set_stream(stream.cuda_stream)
        return case, sim

    if args.profile_case == "stage":
        for prec in ("fp32", "fp64"):
            _, sim = make(prec)
            sim.run(max_step=max(3, args.warmup))
        torch.cuda.synchronize()
        return 0
    if args.profile_case == "corrector":
        # the float Euler path at 256 x 128 x 128 with the 256^3 run's tile k-chunk (12): the
        # same tile shape and grid fill per wave, 0.8 GB on the device
        case = cases.c2_inflow_box(n=(256, 128, 128), flux=args.flux, precision="fp32", seed=4321)
        sim = cases.build_gpu(case, tile_kchunk=12)
        sim.set_stream(stream.cuda_stream)
        sim.run(max_step=max(3, args.warmup))
        torch.cuda.synchronize()
        return 0
    if args.profile_case == "narrow":
        # the float Euler path in tiles 16 cells wide (two rows per warp) at 240 x 128 x 128,
        # k-chunk 32 and the persistent form: what the autotuner picks at 240^3; 0.8 GB
        case = cases.c2_inflow_box(n=(240, 128, 128), flux=args.flux, precision="fp32", seed=4321)
        sim = cases.build_gpu(case, tile_kchunk=32, persistent=True, tile_width=16)
        sim.set_stream(stream.cuda_stream)
        sim.run(max_step=max(3, args.warmup))
        torch.cuda.synchronize()
        return 0
    if args.profile_case == "norms":
        _, sim = make("fp32")
        sim.run(max_step=max(3, args.warmup))
        for _ in range(2):
            sim.residual_norms()
        torch.cuda.synchronize()
        return 0
    if args.profile_case == "mhd":
        for prec in ("fp32", "fp64"):
            sim = cases.build_gpu(cases.orszag_tang(n=(512, 512, 4), precision=prec), fixed_time_step=True,
                                  dt_init=8.0e-5, dt_max=8.0e-5)
            sim.set_stream(stream.cuda_stream)
            sim.run(max_step=max(3, args.warmup))
            sim.close()
        torch.cuda.synchronize()
        return 0
    if args.profile_case == "adjoint":
        adjoint_over_forward(nsteps=10, forms=(("checkpointed", 10),))
        torch.cuda.synchronize()
        return 0
    if args.profile_case == "adjoint_mhd":
        adjoint_mhd_leg(torch.cuda.Stream(), nsteps=10)
        torch.cuda.synchronize()
        return 0

    cells = n ** 3
    results = {}
    sims = {}
    for prec in ("fp32", "fp64"):
        case, sim = make(prec)
        sims[prec] = (case, sim)
        sim.run(max_step=args.warmup)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        sampler = ClockSampler(local)
        with sampler:
            e0.record(stream)
            taken = sim.run(max_step=args.steps)
            e1.record(stream)
            torch.cuda.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1), device="cuda")
        if world > 1:
            dist.barrier()
        results[prec] = dict(ms=ms, taken=taken, clocks=sampler.summary())

    # accuracy of the FP32-flux form against the plain FP64 form after the same steps
    acc_steps = max(args.accuracy_steps, args.warmup + args.steps)
    acc = accuracy_leg({p: sims[p][1] for p in sims}, n, args.flux, acc_steps, stream)
    err = acc["rel_l2_vs_fp64"]

    # roofline of the dominant kernel (corrector stage) of the FP32-flux form, live
    sim32 = sims["fp32"][1]
    st1, st2 = sim32.time_stages(reps=10)
    peak, peak_kind = measured_peaks()
    ach2 = BYTES_STAGE2 * cells / (st2 * 1e-3) / 1e9
    traffic = None
    # ncu DRAM bytes per cell of the corrector (float Euler kernel on decoded primitives),
    # captured on a 256x128x128 case with the same tiles, scaled to this launch's cells
    tf = os.path.join(ROOT, "profiles", "stage_prim_kernel_256x128x128.md")
    if os.path.exists(tf):
        import re
        with open(tf) as f:
            m = re.search(r"stage2_dram_bytes_per_cell:\s*([0-9.]+)", f.read())
        if m:
            traffic = float(m.group(1)) * cells

    # end to end through the public API: host state in, K steps, host state out
    case32, _ = sims["fp32"]
    _, sim_e2e = make("fp32")
    U_host = torch.from_numpy(sim_e2e.get_conserved(0)).pin_memory()
    U_np = U_host.numpy()
    out_np = torch.empty_like(U_host).pin_memory().numpy()   # the result lands in pinned memory too
    sim_e2e.run(max_step=args.warmup)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sim_e2e.set_conserved(0, U_np)
    sim_e2e.run(max_step=args.steps)
    out = sim_e2e.get_conserved(0, out=out_np)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    state_bytes = U_np.nbytes
    e2e_val = world * cells * args.steps / e2e_s / 1e6

    steps = args.steps
    val32 = world * cells * steps / (results["fp32"]["ms"] * 1e-3) / 1e6
    val64 = world * cells * steps / (results["fp64"]["ms"] * 1e-3) / 1e6
    line = {
        "metric": METRIC,
        "value": val32,
        "unit": UNIT,
        "n_gpus": world,
        "steps": steps,
        "warmup": args.warmup,
        "ms_per_step": results["fp32"]["ms"] / steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 flux / f64 state",
        "data": "synthetic (seeded 1% density noise)",
        "config": {"workload": f"M=3 inflow box {n}^3, {args.flux}, l2r2 van Albada, predictor-corrector",
                   "cells": cells, "flux_calculator": args.flux, "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (state 671 MB per buffer)"},
        "fp64_plain": {"value": val64, "ms_per_step": results["fp64"]["ms"] / steps},
        "fp32_over_fp64": val32 / val64,
        "rel_l2_vs_fp64": err,
        "adjoint_over_forward": None,
        "roofline": {"bound": "hbm", "kernel": "stage_prim_kernel<float,2> (corrector)", "achieved": ach2,
                     "peak": peak, "unit": "GB/s", "frac": ach2 / peak, "traffic": traffic,
                     "peak_source": peak_kind, "algorithmic_bytes_per_cell": BYTES_STAGE2,
                     "stage_ms": [st1, st2]},
        "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": state_bytes / steps,
                "d2h_bytes_per_step": (state_bytes + 64 * steps) / steps,
                "how": "gdfv_block_set_conserved from pinned host memory, gdfv_run of all steps, "
                       "gdfv_block_get_conserved back to pinned host memory, wall clock"},
        "gpu_launches": 4 * steps,
        "clocks": results["fp32"]["clocks"],
        "clocks_fp64": results["fp64"]["clocks"],
    }
    line["config"].update(autotune=bool(args.autotune), tile_kchunk=sim32.option("tile_kchunk"),
                          persistent=bool(sim32.option("persistent")), tile_width=sim32.option("tile_width"),
                          tile_rows=sim32.option("tile_rows"),
                          tile_rows_corrector=sim32.option("tile_rows_corrector"))
    line["accuracy"] = acc
    if not args.no_extra:
        for sim in list(sims.values()) + [(None, sim_e2e)]:
            sim[1].close()
        torch.cuda.empty_cache()
        legs = [("adjoint", adjoint_over_forward),
                ("adjoint_mhd", lambda: adjoint_mhd_leg(stream)),
                ("accuracy_other_flux", lambda: accuracy_leg(None, n, "hllc" if args.flux == "ausmdv" else "ausmdv",
                                                             acc_steps, stream)),
                ("multiblock", lambda: multiblock_leg(stream)),
                ("mhd", lambda: mhd_leg(stream)),
                ("chicken_gpu", chicken_gpu_leg)]
        for name, fn in legs:
            try:
                line[name] = fn()
            except Exception as e:  # reported, never required for the throughput line
                line[name] = {"error": f"{type(e).__name__}: {e}"}
            torch.cuda.empty_cache()
        if isinstance(line.get("adjoint"), dict) and "ratio" in line["adjoint"]:
            line["adjoint_over_forward"] = line["adjoint"]["ratio"]
        cg = line.get("chicken_gpu")
        if isinstance(cg, dict) and "value" in cg:   # this library's FP64 form against the reference's GPU code
            cg["fp64_plain_over_chicken_gpu_per_step"] = line["fp64_plain"]["value"] / cg["value"]
            cg["fp64_plain_over_chicken_gpu_per_stage"] = 2 * line["fp64_plain"]["value"] / cg["value_per_stage"]
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the reference's own CPU build when present (kind "reference"), the oracle port beside it
        try:
            ref = chicken_baseline(10, 2)
        except Exception as e:  # the baseline is reported, never required
            ref = None
            line["cpu_baseline_reference_error"] = str(e)
        try:
            port = cpu_oracle_baseline()
        except Exception as e:
            port = {"error": str(e)}
        line["cpu_baseline"] = ref["cpu_baseline"] if ref else port
        line["cpu_baseline_port"] = port
    if world > 1:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
