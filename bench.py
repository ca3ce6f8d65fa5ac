#!/usr/bin/env python
"""Benchmark of the MPulse time-stepping path on B200.

Workload: PLRC + Kerr + CPML at 256 x 256 x 512 cells (two-pole Lorentz medium
with chi3 E0^2 = 0.01 for z >= 64, 12-cell CPML on all six faces, focused
Gaussian pulse injected by the paraxial short-pulse closed form), FP32 device
state.  One "step" is one MPulse time step (E half + B half) over the whole
grid.  The metric is Gcell-updates/s = nx ny nz x steps / time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`value` is timed with CUDA events on the simulation's stream, state resident in
HBM (4.7 GB, larger than the 126 MB L2, so no L2 flush is needed).  `e2e` is the
same metric through the C ABI with host buffers: upload of the six fields from
pinned host memory, K steps, download of E, all inside the timed region.
The FP64 form runs the same steps beside it, and the relative L2 error of the
FP32 fields against it is reported.  With N > 1 every rank runs its own
independent simulation (replicas only: the path is not sharded).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from mpulse_b200 import abi, configs  # noqa: E402

WORKLOAD = dict(nx=256, ny=256, nz=512)
WORKLOAD_NAME = "plrc_kerr_cpml_focused_256x256x512"
METRIC = "Gcell-updates/s FP32 vs FP64 at rel-L2<=1e-5; adjoint/forward time ratio"
UNIT = "Gcell-updates/s"
# Process::time at which the timed steps start: the pulse is being injected then.
START_TIME = 700


def bench_config(precision: int) -> abi.Config:
    return configs.c3_plrc_kerr(precision=precision, **WORKLOAD)


def algorithmic_bytes(cfg: abi.Config, elem: int) -> dict:
    """Algorithmic HBM bytes per step: every state element read once and written
    once; neighbours, coefficient lines and source planes are free.
        step:   s [12 N + 12 P N_med + 8 N_cpml]
        E half: s [ 9 N + 12 P N_med + 4 N_cpml]   (E r/w, B r, psi r/w, psi_E r/w)
        B half: s [ 9 N + 4 N_cpml]                 (B r/w, E r, psi_H r/w)
    N_cpml counts face-slab cells per face (overlapping corners once per face)."""
    N = cfg.nx * cfg.ny * cfg.nz
    P = sum(1 for n in range(3) if cfg.poles[n].eps != 0)
    z0 = max(cfg.medium_z0, 1)
    z1 = min(cfg.medium_z1, cfg.nz)
    Nmed = max(0, z1 - z0 + 1) * cfg.nx * cfg.ny
    d = cfg.cpml_d
    if cfg.cpml == abi.MP_CPML_ALL:
        Ncpml = d * (2 * cfg.ny * cfg.nz + 2 * cfg.nx * cfg.nz + 2 * cfg.nx * cfg.ny)
    elif cfg.cpml == abi.MP_CPML_Z:
        Ncpml = d * 2 * cfg.nx * cfg.ny
    else:
        Ncpml = 0
    return {
        "step": elem * (12 * N + 12 * P * Nmed + 8 * Ncpml),
        "e_half": elem * (9 * N + 12 * P * Nmed + 4 * Ncpml),
        "b_half": elem * (9 * N + 4 * Ncpml),
        "N": N, "P": P, "N_med": Nmed, "N_cpml": Ncpml,
    }


def measured_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return {"hbm_gbs": d.get("hbm_gbs", 6650.0), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(prefix="clk_", suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.3)  # let nvidia-smi start before the timed region
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def follow_trace(sim, axis, z_start: int, steps: int = 16) -> list:
    """FollowMax::calculate (followmax.cpp:73-113) of Ex along z through the
    column `axis`, after each of `steps` steps (mp_follow_max)."""
    ip, out = z_start, []
    for _ in range(steps):
        sim.step(1)
        ip, x = sim.follow_max("Ex", 2, (axis[0], axis[1], ip), ip)
        out.append(x)
    return out


def time_steps(sim, torch, steps: int, stream) -> tuple[float, int]:
    """Device time (s) of `steps` steps with CUDA events on the sim's stream."""
    L0 = sim.launches
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record(stream)
    sim.step_async(steps)
    stop.record(stream)
    torch.cuda.synchronize()
    sim.check_status()
    return start.elapsed_time(stop) / 1e3, sim.launches - L0


def max_over_ranks(t: float, dist, device: str) -> float:
    """The largest of the ranks' device times (the job's time); `dist` is
    torch.distributed or None for one process."""
    if dist is None:
        return t
    import torch
    x = torch.tensor([t], device=device, dtype=torch.float64)
    dist.all_reduce(x, op=dist.ReduceOp.MAX)
    return float(x.item())


def replica_value(cells: int, steps: int, t_max: float, world: int) -> float:
    """Whole-job Gcell-updates/s: every rank runs its own replica of the
    workload (weak scaling), timed by the slowest rank."""
    return world * cells * steps / t_max / 1e9


def run_ours(args) -> dict:
    import torch
    from mpulse_b200 import runtime

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local_rank))
    else:
        torch.cuda.set_device(0)

    cfg = bench_config(abi.MP_FP32)
    cfg.device = local_rank
    stream = torch.cuda.Stream()
    sim = runtime.Simulation(cfg)
    sim.set_stream(stream.cuda_stream)
    sim.time = START_TIME
    # warm-up
    sim.step(args.warmup)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    barrier()
    with ClockSampler(local_rank) as clk:
        dt_dev, launches = time_steps(sim, torch, args.steps, stream)
    clocks = clk.summary()
    barrier()
    t_max = max_over_ranks(dt_dev, dist, "cuda")
    cells = cfg.nx * cfg.ny * cfg.nz
    value = replica_value(cells, args.steps, t_max, world)
    # FP32 state after warmup + steps, compared below with the FP64 form
    fp32_state = {n: sim.download(n) for n in ("Ex", "Ey", "Ez")}
    # FollowMax of Ex along z through the beam axis, over the next steps
    axis = (cfg.nx // 2, cfg.ny // 2)
    z_start = int(np.argmax(np.abs(fp32_state["Ex"][1:-1, axis[1] - 1, axis[0] - 1]))) + 1
    trace32 = follow_trace(sim, axis, z_start)

    # per-kernel device times (CUDA events around each launch, further steps)
    kt = sim.kernel_times(max(3, min(args.steps, 10)))
    alg = algorithmic_bytes(cfg, 4)
    peaks = measured_peaks()
    e_ms = kt["e_half_ms"]
    achieved = alg["e_half"] / (e_ms / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic_e_half.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            traffic = json.load(f).get("bytes_per_launch")
    roofline = {"bound": "hbm", "kernel": "e_half_kernel<float,PLRC_NONLIN,2>", "achieved": round(achieved, 1),
                "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": round(achieved / peaks["hbm_gbs"], 4),
                "traffic": traffic, "peak_source": peaks["source"],
                "algorithmic_bytes_per_launch": alg["e_half"], "launch_ms": round(e_ms, 4)}
    step_achieved = alg["step"] / (t_max / args.steps) / 1e9
    step_roofline = {"achieved": round(step_achieved, 1), "frac": round(step_achieved / peaks["hbm_gbs"], 4),
                     "algorithmic_bytes_per_step": alg["step"], "unit": "GB/s"}

    # FP64 form on the same steps, and the FP32 error against it
    sim.close()
    torch.cuda.empty_cache()
    cfg64 = bench_config(abi.MP_FP64)
    cfg64.device = local_rank
    sim64 = runtime.Simulation(cfg64)
    sim64.set_stream(stream.cuda_stream)
    sim64.time = START_TIME
    sim64.step(args.warmup)
    dt64, _ = time_steps(sim64, torch, args.steps, stream)
    fp64_state = {n: sim64.download(n) for n in ("Ex", "Ey", "Ez")}
    trace64 = follow_trace(sim64, axis, z_start)
    sim64.close()
    num = sum(float(np.sum((fp32_state[n] - fp64_state[n]) ** 2)) for n in fp32_state)
    den = sum(float(np.sum(fp64_state[n] ** 2)) for n in fp64_state)
    rel = math.sqrt(num / den) if den > 0 else None
    value64 = world * cells * args.steps / dt64 / 1e9

    # end to end through the C ABI with host buffers
    e2e = run_e2e(args, torch, stream, local_rank)
    adjoint = run_adjoint(local_rank) if rank == 0 else None
    others = run_other_configs(local_rank, torch, stream) if rank == 0 else None

    out = {
        "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(t_max / args.steps * 1e3, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD_NAME, "grid": [cfg.nx, cfg.ny, cfg.nz], "solver": "fdtd-plrc-nonlin",
                   "poles": 2, "cpml": "all faces, d=12", "source": "short_pulse_inject (focused, waist 2 um)",
                   "start_time": START_TIME, "parallelism": f"replicas{world}",
                   "l2": "state 4.7 GB > 126 MB L2, no flush needed"},
        "fp64": {"value": round(value64, 4), "unit": UNIT, "ms_per_step": round(dt64 / args.steps * 1e3, 4)},
        "fp32_over_fp64": round(value / value64, 3) if value64 > 0 else None,
        "rel_l2_fp32_vs_fp64": rel,
        "followmax": {"field": "Ex", "dim": "z", "line_xy": list(axis), "steps": len(trace32),
                      "fp32": [round(x, 4) for x in trace32], "fp64": [round(x, 4) for x in trace64],
                      "max_abs_diff": float(np.max(np.abs(np.array(trace32) - np.array(trace64))))},
        "adjoint_forward_ratio": adjoint["fp32"]["ratio"] if adjoint else None,
        "adjoint": adjoint,
        "other_workloads": others,
        "roofline": roofline, "step_roofline": step_roofline,
        "kernel_ms": kt,
        "e2e": e2e,
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    if args.cpu_baseline and rank == 0 and world == 1:
        out["cpu_baseline"] = cpu_baseline_sample(args)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return out if rank == 0 else None


def run_other_configs(local_rank: int, torch, stream) -> dict:
    """The parity workloads beside the headline one, FP32 and FP64 forms
    (device time of the step loop, CUDA events): the 64^3 vacuum pulse
    (pulse_init start, 400 steps) and the 128^3 linear PLRC workload
    (plane_gauss_inject, 1000 steps).  The FP32 error of E against the FP64
    form is taken every 100 steps of a second, untimed pair of runs: relative
    L2 at the end and when the FP64 field norm peaks, and the final error over
    that peak norm (late in these runs the pulse has left through the CPML
    and the field that remains is small, so the final relative error alone
    measures residue)."""
    from mpulse_b200 import runtime
    out = {}
    for name, make, steps, init in (
            ("c1_vacuum_pulse_64^3_400steps", configs.c1_vacuum_pulse, 400, configs.c1_initial_fields),
            ("c2_linear_plrc_128^3_1000steps", configs.c2_linear_plrc, 1000, None)):
        res, sims = {}, {}
        for prec, tag in ((abi.MP_FP32, "fp32"), (abi.MP_FP64, "fp64")):
            cfg = make(prec)
            cfg.device = local_rank
            with runtime.Simulation(cfg) as g:
                g.set_stream(stream.cuda_stream)
                if init is not None:
                    for n, v in init(cfg).items():
                        g.upload(n, v)
                g.step(1)  # first launches out of the timed region
                dt, _ = time_steps(g, torch, steps - 1, stream)
            res[tag] = round(cfg.nx * cfg.ny * cfg.nz * (steps - 1) / dt / 1e9, 3)
            sims[tag] = runtime.Simulation(cfg)
            if init is not None:
                for n, v in init(cfg).items():
                    sims[tag].upload(n, v)
        at_peak, peak, diff, norm = None, 0.0, 0.0, 0.0
        for _ in range(steps // 100):
            for g in sims.values():
                g.step(100)
            e32 = [sims["fp32"].download(n) for n in ("Ex", "Ey", "Ez")]
            e64 = [sims["fp64"].download(n) for n in ("Ex", "Ey", "Ez")]
            diff = math.sqrt(sum(float(np.sum((a - b) ** 2)) for a, b in zip(e32, e64)))
            norm = math.sqrt(sum(float(np.sum(b ** 2)) for b in e64))
            if norm > peak:
                peak = norm
                at_peak = diff / norm
        for g in sims.values():
            g.close()
        res["unit"] = UNIT
        res["rel_l2_fp32_vs_fp64_final"] = diff / norm if norm > 0 else None
        res["rel_l2_fp32_vs_fp64_at_peak_norm"] = at_peak
        res["final_error_over_peak_norm"] = diff / peak if peak > 0 else None
        res["final_norm_over_peak_norm"] = norm / peak if peak > 0 else None
        out[name] = res
    return out


def run_adjoint(local_rank: int) -> dict:
    """The adjoint workload (96^3, single-pole medium, 32^3 design region,
    1500 steps, |E|^2 monitor objective): wall time of the forward run that
    computes J (mp_objective) and of mp_adjoint (forward with checkpoints +
    reverse pass), best of three; FP32 with a checkpoint every 50 steps (the
    workload's schedule) and with the whole E history kept, and the FP32
    gradient against the FP64 one."""
    from mpulse_b200 import runtime

    out = {"workload": "adjoint_plrc_96^3_design32^3_1500steps", "unit": "s"}
    grads = {}
    for prec, tag in ((abi.MP_FP32, "fp32"), (abi.MP_FP64, "fp64")):
        cfg, des, adj = configs.c4_adjoint(prec)
        cfg.device = local_rank
        full = abi.adjoint_config(adj.kind, list(adj.box), adj.steps, checkpoint_every=adj.steps)

        def fresh():
            g = runtime.Simulation(cfg)
            for k, v in des.items():
                g.upload_design(k, v)
            g.sync()
            return g

        def timed(fn):
            best, res = None, None
            for _ in range(3):
                with fresh() as g:
                    t0 = time.perf_counter()
                    res = fn(g)
                    t = time.perf_counter() - t0
                best = t if best is None else min(best, t)
            return best, res

        warm = abi.adjoint_config(adj.kind, list(adj.box), 60, checkpoint_every=20)
        with fresh() as g:
            g.adjoint(warm)
        fwd, J = timed(lambda g: g.objective(adj))
        t_adj, (Ja, gr) = timed(lambda g: g.adjoint(adj))
        t_full, _ = timed(lambda g: g.adjoint(full))
        grads[tag] = gr["DesignEps"]
        out[tag] = {"forward_s": round(fwd, 4), "adjoint_s": round(t_adj, 4),
                    "ratio": round(t_adj / fwd, 3), "checkpoint_every": adj.checkpoint_every,
                    "adjoint_full_history_s": round(t_full, 4), "ratio_full_history": round(t_full / fwd, 3),
                    "J": J}
    g32, g64 = grads["fp32"], grads["fp64"]
    out["grad_rel_l2_fp32_vs_fp64"] = float(np.linalg.norm(g32 - g64) / np.linalg.norm(g64))
    return out


def run_adjoint_profile(args) -> dict:
    """The adjoint workload only, FP32, args.steps steps with a checkpoint
    every args.checkpoint steps: mp_objective, then mp_adjoint (for ncu
    captures of the adjoint kernels)."""
    from mpulse_b200 import runtime
    cfg, des, adj = configs.c4_adjoint(abi.MP_FP32)
    a = abi.adjoint_config(adj.kind, list(adj.box), args.steps, checkpoint_every=args.checkpoint)
    out = {"adjoint_profile_run": True, "steps": args.steps, "checkpoint_every": args.checkpoint}
    with runtime.Simulation(cfg) as g:
        for k, v in des.items():
            g.upload_design(k, v)
        out["J_objective"] = g.objective(a)
    with runtime.Simulation(cfg) as g:
        for k, v in des.items():
            g.upload_design(k, v)
        out["J_adjoint"], _ = g.adjoint(a)
    return out


def run_adjoint_large(args) -> dict:
    """The large nonlinear adjoint workload (512 x 512 x 768, Sz objective,
    FP32) for args.steps steps: forward (mp_objective) and mp_adjoint under a
    memory budget of args.budget_gb GB for checkpoints and history (the
    library picks the schedule); then the FP32 gradient against the FP64
    adjoint on a 64^3 crop of the workload (16^3 design region, 320 steps)."""
    from mpulse_b200 import runtime
    out = {"adjoint_large_run": True, "steps": args.steps, "budget_gb": args.budget_gb}
    cfg, des, adj = configs.c5_adjoint(abi.MP_FP32, steps=args.steps)
    adj.mem_budget = args.budget_gb * 1e9
    cells = cfg.nx * cfg.ny * cfg.nz

    def fresh(c, d):
        g = runtime.Simulation(c)
        for k, v in d.items():
            g.upload_design(k, v)
        g.sync()
        return g

    with fresh(cfg, des) as g:
        t0 = time.perf_counter()
        out["J_forward"] = g.objective(adj)
        out["forward_s"] = time.perf_counter() - t0
    out["forward_gcells"] = cells * args.steps / out["forward_s"] / 1e9
    with fresh(cfg, des) as g:
        t0 = time.perf_counter()
        out["J_adjoint"], gr = g.adjoint(adj)
        out["adjoint_s"] = time.perf_counter() - t0
    out["ratio"] = out["adjoint_s"] / out["forward_s"]
    out["grad_norm_eps"] = float(np.linalg.norm(gr["DesignEps"]))
    # 64^3 crop: FP32 against FP64
    grads = {}
    for prec in (abi.MP_FP32, abi.MP_FP64):
        c2, d2, a2 = configs.c5_adjoint(prec, nx=64, ny=64, nz=64, steps=320, design=(16, 16, 16), design_z0=24,
                                         sz_plane=52, src_d=6, cpml_d=6, medium_z0=10)
        a2.mem_budget = 0
        with fresh(c2, d2) as g:
            _, grads[prec] = g.adjoint(a2)
    out["crop_grad_rel_l2_fp32_vs_fp64"] = {
        k: float(np.linalg.norm(grads[abi.MP_FP32][k] - grads[abi.MP_FP64][k]) / np.linalg.norm(grads[abi.MP_FP64][k]))
        for k in ("DesignEps", "DesignChiScale")}
    return out


def run_profile(args) -> dict:
    """FP32 workload only: warm-up, then the timed steps; no other kernels."""
    import torch
    from mpulse_b200 import runtime
    torch.cuda.set_device(0)
    cfg = bench_config(abi.MP_FP32)
    stream = torch.cuda.Stream()
    sim = runtime.Simulation(cfg)
    sim.set_stream(stream.cuda_stream)
    sim.time = START_TIME
    sim.step(args.warmup)
    dt, launches = time_steps(sim, torch, args.steps, stream)
    cells = cfg.nx * cfg.ny * cfg.nz
    kt = sim.kernel_times(5)
    sim.close()
    return {"profile_run": True, "grid": [cfg.nx, cfg.ny, cfg.nz], "steps": args.steps,
            "value": cells * args.steps / dt / 1e9, "unit": UNIT, "gpu_launches": launches, "kernel_ms": kt}


def run_e2e(args, torch, stream, local_rank) -> dict:
    from mpulse_b200 import runtime
    cfg = bench_config(abi.MP_FP32)
    cfg.device = local_rank
    count = cfg.field_count()
    host_in = {n: torch.zeros(count, dtype=torch.float64, pin_memory=True).numpy() for n in abi.FIELD_NAMES}
    host_out = {n: torch.zeros(count, dtype=torch.float64, pin_memory=True).numpy() for n in ("Ex", "Ey", "Ez")}
    sim = runtime.Simulation(cfg)
    sim.set_stream(stream.cuda_stream)
    sim.time = START_TIME
    sim.step(1)  # first launch out of the timed region
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for n in abi.FIELD_NAMES:
        sim.upload(n, host_in[n])
    sim.step(args.steps)
    for n in ("Ex", "Ey", "Ez"):
        sim.download(n, host_out[n])
    t1 = time.perf_counter()
    sim.close()
    cells = cfg.nx * cfg.ny * cfg.nz
    return {"value": round(cells * args.steps / (t1 - t0) / 1e9, 4), "unit": UNIT,
            "h2d_bytes_per_step": int(6 * count * 8 / args.steps), "d2h_bytes_per_step": int(3 * count * 8 / args.steps),
            "what": "mp_upload x6 (pinned double) + mp_step(K) + mp_download x3, wall clock"}


# ---------------------------------------------------------------------------
# The reference on the host cores.

def _ref_binary():
    for name in ("mpulse_ref_fast", "mpulse_ref"):
        p = os.path.join(ROOT, "oracle", "_ref", name)
        if os.path.exists(p):
            return p
    return None


def reference_slabs(steps: int, warmup: int, procs: int) -> dict:
    """Runs the reference build on the bench workload split into `procs`
    independent z-slabs (MPulse's own slab decomposition without the halo
    exchange, one process per core, as its MPI build would run them) for
    warmup + steps steps, and returns the aggregate rate of the timed steps."""
    from oracle import pyoracle
    binary = _ref_binary()
    cfg = bench_config(abi.MP_FP64)
    nz_slab = max(2 * cfg.cpml_d, cfg.nz // procs)
    procs = max(1, cfg.nz // nz_slab)
    tmp = tempfile.mkdtemp(prefix="mpref_bench_")
    runs = []
    for p in range(procs):
        c = bench_config(abi.MP_FP64)
        c.nz = nz_slab
        c.medium_z0 = 0 if p > 0 else cfg.medium_z0
        c.medium_z1 = nz_slab + 1
        d = os.path.join(tmp, f"r{p}")
        os.makedirs(d)
        with open(os.path.join(d, "setup.dat"), "w") as f:
            f.write(pyoracle.setup_text(c, warmup + steps))
        env = dict(os.environ, MPULSE_REF_WARMUP=str(warmup))
        runs.append((subprocess.Popen([binary, os.path.join(d, "setup.dat"), d], stdout=subprocess.PIPE,
                                      stderr=subprocess.DEVNULL, env=env, text=True), c))
    secs, cells, rates = [], 0, []
    for pr, c in runs:
        outp, _ = pr.communicate()
        if pr.returncode != 0:
            raise RuntimeError("reference run failed")
        r = json.loads(outp.strip().splitlines()[-1])
        secs.append(r["seconds"])
        cells += r["cells"]
        rates.append(r["cells"] * steps / r["seconds"] / 1e9)
    t = max(secs)
    return {"value": cells * steps / t / 1e9, "procs": procs, "cells": cells, "seconds": t, "nz_slab": nz_slab,
            "per_core": float(np.median(rates))}


def cpu_baseline_sample(args) -> dict:
    """Bounded CPU baseline for the headline line: the reference build on the
    host cores for 2 timed steps of the full workload, split into z-slabs."""
    if _ref_binary() is None:
        return cpu_baseline_port()
    procs = max(1, min(os.cpu_count() or 1, 64))
    r = reference_slabs(steps=2, warmup=1, procs=procs)
    return {"value": round(r["value"], 6), "unit": UNIT, "cores": r["procs"], "kind": "reference",
            "sample": f"MPulse reference build (-O3), full 256x256x512 workload as {r['procs']} independent "
                      f"z-slabs of {r['nz_slab']} planes, 1 warm-up + 2 timed steps",
            "per_core_value": round(r["per_core"], 6),
            "per_core": "median rate of one slab process (the reference is single-threaded), measured while all ran"}


def cpu_baseline_port() -> dict:
    from oracle import pyoracle
    c = bench_config(abi.MP_FP64)
    c.nz = 32
    c.medium_z0 = 0
    o = pyoracle.OracleSim(c)
    o.time = START_TIME
    t0 = time.perf_counter()
    o.step(2)
    t = time.perf_counter() - t0
    return {"value": round(c.nx * c.ny * c.nz * 2 / t / 1e9, 6), "unit": UNIT, "cores": 1, "kind": "port",
            "sample": "C oracle, 256x256x32 slab of the workload, 2 steps"}


def run_reference_arm(args) -> dict | None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    if _ref_binary() is None:
        return {"impl": "reference", "unavailable": "reference build missing (make -C oracle ref)"}
    procs = max(1, min(os.cpu_count() or 1, 64))
    t0 = time.perf_counter()
    r = reference_slabs(steps=args.steps, warmup=args.warmup, procs=procs)
    wall = time.perf_counter() - t0
    v = round(r["value"], 6)
    sample = (f"MPulse reference build (-O3), the {WORKLOAD_NAME} workload as {r['procs']} independent z-slab "
              f"processes of {r['nz_slab']} planes, {args.warmup} warm-up + {args.steps} timed steps")
    return {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": 0, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(r["seconds"] / args.steps * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD_NAME, "grid": [256, 256, 512], "parallelism": f"{r['procs']} processes"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": r["procs"], "kind": "reference", "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": round(wall, 2),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--profile-only", action="store_true",
                    help="only the FP32 warm-up and timed steps (for ncu captures)")
    ap.add_argument("--nz", type=int, default=None, help="override nz (smaller case for ncu --set full)")
    ap.add_argument("--adjoint-only", action="store_true",
                    help="only mp_objective + mp_adjoint of the adjoint workload for --steps steps (ncu captures)")
    ap.add_argument("--checkpoint", type=int, default=50, help="checkpoint interval of --adjoint-only")
    ap.add_argument("--adjoint-large", action="store_true",
                    help="the 512x512x768 nonlinear adjoint workload for --steps steps (minutes)")
    ap.add_argument("--budget-gb", type=float, default=120.0, help="checkpoint budget of --adjoint-large")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.nz:
        WORKLOAD["nz"] = args.nz
    if args.adjoint_large:
        out = run_adjoint_large(args)
    elif args.adjoint_only:
        out = run_adjoint_profile(args)
    elif args.profile_only:
        out = run_profile(args)
    else:
        out = run_reference_arm(args) if args.impl == "reference" else run_ours(args)
    if out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
