#!/usr/bin/env python
"""Benchmark of the MPulse time-stepping path on B200.

Workload: PLRC + Kerr + CPML at 256 x 256 x 512 cells (two-pole Lorentz medium
with chi3 E0^2 = 0.01 for z >= 64, 12-cell CPML on all six faces, focused
Gaussian pulse injected by the paraxial short-pulse closed form), FP32 device
state, dt = 0.45 dx / c.  One "step" is one MPulse time step (E half + B half)
over the whole grid.  The metric is Gcell-updates/s = nx ny nz x steps / time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

The FP32 and FP64 forms run side by side from time 0 (both contexts live at
once).  An untimed pre-roll of PREROLL_STEPS steps brings the pulse into the
Kerr medium; after W warm-up steps, `value` times K steps of the FP32 form with
CUDA events on the simulation's stream (state 4.7 GB, larger than the 126 MB
L2, so no L2 flush is needed), plus the device time of the injection planes of
those K steps, measured on their own and added pro rata (the planes are
computed ahead in batches on a second stream and overlap the step kernels;
the addition gives no credit for that overlap).  The E half-step kernel counts
its Kerr solves and Newton iterations on the device during the timed steps.
`e2e` is the same metric through the C ABI with host buffers: upload of the
six fields from pinned host memory, K steps, download of E, all inside the
timed region.  Both forms then continue to step 4000 (the workload's run
length), with FollowMax (followmax.cpp:73-113) of Ex along the beam axis after
every step and the relative L2 error of E (FP32 against FP64) and the peak
|E|^2 every 50 steps.  With N > 1 every rank runs its own independent
simulation (replicas only: the path is not sharded).
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
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from mpulse_b200 import abi, configs  # noqa: E402

WORKLOAD = dict(nx=256, ny=256, nz=512)
WORKLOAD_NAME = "plrc_kerr_cpml_focused_256x256x512"
METRIC = "Gcell-updates/s FP32 vs FP64 at rel-L2<=1e-5; adjoint/forward time ratio"
UNIT = "Gcell-updates/s"
# Untimed steps from time 0 before the warm-up.  The pulse (20 fs FWHM, field
# 1/e half-width T = 5.09 um / c) peaks on the injection plane z = 20 at
# t = 3 T (848 steps of dt = 0.018 um / c), reaches the medium at z = 64 about
# 98 steps later and then moves about one cell per 3.3 steps (group index about
# 1.47): at step 1100 its peak is some 47 cells into the Kerr medium, and the
# field is non-zero in every medium cell.
PREROLL_STEPS = 1100
ACCURACY_STEPS = 4000     # run length of the workload
RECORD_EVERY = 50         # FP32-vs-FP64 error and peak |E|^2 sampled this often


def workload_config_keys(cfg: abi.Config) -> dict:
    """The `config` object of both arms' lines: the workload itself."""
    return {"workload": WORKLOAD_NAME, "grid": [cfg.nx, cfg.ny, cfg.nz], "solver": "fdtd-plrc-nonlin",
            "poles": 2, "chi3_E0^2": cfg.chi, "cpml": f"all faces, d={cfg.cpml_d}",
            "source": "short_pulse_inject (focused, waist 2 um at z=200, 20 fs, injected at z=20)",
            "dx_um": cfg.dx,
            "dt": f"{configs.MEDIUM_COURANT} dx/c = {cfg.dt:g} um/c (0.5 dx/c amplifies grid noise with this "
                  f"medium in the reference scheme as well; pinned by tests/test_stability.py)",
            "l2": "state 4.7 GB (FP32) > 126 MB L2, no flush needed"}


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


def device_array(sim, name: str, torch):
    """A torch view (no copy) of one field's device array, for the FP32-vs-FP64
    comparisons of the measurement (mp_device_field)."""
    ptr, count, elem = sim.device_field(name)

    class _View:
        __cuda_array_interface__ = {"shape": (count,), "typestr": "<f4" if elem == 4 else "<f8",
                                    "data": (ptr, False), "strides": None, "version": 2}

    return torch.as_tensor(_View(), device="cuda")


class PairRun:
    """The FP32 and FP64 forms of the workload stepped in lockstep.  After every
    step of advance() it runs FollowMax (mp_follow_max, followmax.cpp:73-113)
    of Ex along z through the beam axis on both, from the injection plane on;
    every RECORD_EVERY steps it records the relative L2 error of E (FP32
    against FP64, over all stored cells), the FP64 field norm and the peak
    |E|^2 of both forms (device reductions in FP64)."""

    def __init__(self, sim32, sim64, cfg, torch):
        self.s32, self.s64, self.torch = sim32, sim64, torch
        self.axis = (cfg.nx // 2, cfg.ny // 2)
        self.start = cfg.sources[0].distance
        self.ip = {32: self.start, 64: self.start}
        self.pos = {32: float(self.ip[32]), 64: float(self.ip[64])}
        self.records = []

    def follow(self):
        for tag, sim in ((32, self.s32), (64, self.s64)):
            self.ip[tag], self.pos[tag] = sim.follow_max("Ex", 2, (self.axis[0], self.axis[1], self.ip[tag]),
                                                         self.ip[tag])

    def compare(self) -> dict:
        torch = self.torch
        torch.cuda.synchronize()
        e32 = [device_array(self.s32, n, torch) for n in ("Ex", "Ey", "Ez")]
        e64 = [device_array(self.s64, n, torch) for n in ("Ex", "Ey", "Ez")]
        diff = sum(float(torch.sum((a.double() - b) ** 2)) for a, b in zip(e32, e64))
        norm = sum(float(torch.sum(b * b)) for b in e64)
        i32 = float(torch.max(sum(a.double() ** 2 for a in e32)))
        i64 = float(torch.max(sum(b * b for b in e64)))
        return {"diff": math.sqrt(diff), "norm": math.sqrt(norm), "peak_I32": i32, "peak_I64": i64}

    def record(self):
        c = self.compare()
        self.records.append({"step": self.s32.time, "rel_l2": c["diff"] / c["norm"] if c["norm"] > 0 else None,
                             "norm": c["norm"], "err": c["diff"], "peak_I32": c["peak_I32"], "peak_I64": c["peak_I64"],
                             "follow32": self.pos[32], "follow64": self.pos[64]})

    def advance(self, steps: int):
        for _ in range(steps):
            self.s32.step_async(1)
            self.s64.step_async(1)
            self.follow()
            if self.s32.time % RECORD_EVERY == 0:
                self.s32.check_status()
                self.s64.check_status()
                self.record()

    def summary(self) -> dict:
        """The error of the FP32 form is measured against the FP64 form's field
        norm at its largest over the run (the pulse in the domain): late in the
        run the pulse has left through the CPML and the field that remains is
        a residue of 1e-4 of that norm, so its own relative error measures
        rounding noise on the residue, not the field.  Both are reported; the
        rel-L2 <= 1e-5 bar applies to the error over the peak norm and to the
        relative error while the field norm is at least 1% of its peak."""
        recs = [r for r in self.records if r["norm"] > 0]
        peak = max(recs, key=lambda r: r["norm"])
        last = self.records[-1]
        live = [r for r in recs if r["norm"] >= 0.01 * peak["norm"]]
        return {
            "steps": last["step"], "record_every": RECORD_EVERY,
            "error_over_peak_norm_max": max(r["err"] for r in self.records) / peak["norm"],
            "final_error_over_peak_norm": last["err"] / peak["norm"],
            "rel_l2_fp32_vs_fp64_max_while_norm_ge_1pct_of_peak": max(r["rel_l2"] for r in live),
            "steps_with_norm_ge_1pct_of_peak": [live[0]["step"], live[-1]["step"]],
            "rel_l2_fp32_vs_fp64_at_peak_norm": peak["rel_l2"], "peak_norm_step": peak["step"],
            "rel_l2_fp32_vs_fp64_final": last["rel_l2"],
            "final_norm_over_peak_norm": last["norm"] / peak["norm"],
            "rel_l2_trace": [[r["step"], r["rel_l2"], r["norm"] / peak["norm"]] for r in self.records],
            "followmax": {"field": "Ex", "dim": "z", "line_xy": list(self.axis), "every_step": True,
                          "start_z": self.start,
                          "max_abs_diff_cells_while_norm_ge_1pct_of_peak":
                              max(abs(r["follow32"] - r["follow64"]) for r in live),
                          "max_abs_diff_cells": max(abs(r["follow32"] - r["follow64"]) for r in self.records),
                          "trace": [[r["step"], round(r["follow32"], 4), round(r["follow64"], 4)]
                                    for r in self.records]},
            "peak_intensity": {"what": "max over the grid of Ex^2 + Ey^2 + Ez^2",
                               "max_rel_diff": max(abs(r["peak_I32"] - r["peak_I64"]) / r["peak_I64"]
                                                   for r in recs if r["peak_I64"] > 0),
                               "trace": [[r["step"], r["peak_I32"], r["peak_I64"]] for r in self.records]},
        }


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
    cfg64 = bench_config(abi.MP_FP64)
    cfg64.device = local_rank
    stream = torch.cuda.Stream()
    sim = runtime.Simulation(cfg)
    sim64 = runtime.Simulation(cfg64)
    for g in (sim, sim64):
        g.set_stream(stream.cuda_stream)
    pair = PairRun(sim, sim64, cfg, torch)
    # untimed pre-roll from time 0, then the warm-up
    pair.advance(args.preroll)
    pair.advance(args.warmup)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    cells = cfg.nx * cfg.ny * cfg.nz
    sim.kerr_counts()  # reset the device counters
    barrier()
    with ClockSampler(local_rank) as clk:
        dt_dev, launches = time_steps(sim, torch, args.steps, stream)
    clocks = clk.summary()
    kerr_solves, kerr_iters = sim.kerr_counts()
    barrier()
    t0_window = sim.time - args.steps
    sim64.kerr_counts()
    dt64, _ = time_steps(sim64, torch, args.steps, stream)
    kerr64 = sim64.kerr_counts()
    pair.follow()
    state = pair.compare()
    # per-kernel device times (CUDA events around each launch, further steps,
    # the same number on both forms so they stay in lockstep)
    nkt = max(3, min(args.steps, 10))
    kt = sim.kernel_times(nkt)
    kt64 = sim64.kernel_times(nkt)
    pair.follow()
    # the injection planes of the timed steps were computed before the window:
    # their device time, pro rata
    src_s = args.steps * kt["sources_ms"] / 1e3
    src64_s = args.steps * kt64["sources_ms"] / 1e3
    t_max = max_over_ranks(dt_dev + src_s, dist, "cuda")
    value = replica_value(cells, args.steps, t_max, world)
    value64 = world * cells * args.steps / (dt64 + src64_s) / 1e9

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
                     "algorithmic_bytes_per_step": alg["step"], "unit": "GB/s",
                     "what": "step bytes / (window + sources pro rata) per step"}

    # end to end through the C ABI with host buffers (FP32 form), then the same
    # steps on the FP64 form to keep the pair in lockstep
    e2e = run_e2e(args, torch, sim, cfg)
    sim64.step(args.steps)
    pair.follow()
    # both forms on to the end of the workload's run
    pair.advance(max(0, ACCURACY_STEPS - sim.time))
    accuracy = pair.summary()
    sim.close()
    sim64.close()
    torch.cuda.empty_cache()

    adjoint = run_adjoint(local_rank) if rank == 0 else None
    others = run_other_configs(local_rank, torch, stream) if rank == 0 else None

    n_med = alg["N_med"]
    out = {
        "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(t_max / args.steps * 1e3, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config_keys(cfg),
        "parallelism": f"replicas{world}",
        "state": {"what": f"untimed pre-roll of {args.preroll} steps from time 0 and {args.warmup} warm-up steps "
                          f"(FP32 and FP64 side by side): the pulse is in the Kerr medium",
                  "first_timed_step": t0_window,
                  "kerr_solves_per_step": kerr_solves / args.steps,
                  "newton_iterations_per_solve": kerr_iters / kerr_solves if kerr_solves else None,
                  "medium_cells": n_med, "kerr_solves_over_medium_cells": kerr_solves / args.steps / n_med,
                  "fp64_kerr_solves_per_step": kerr64[0] / args.steps},
        "window": {"device_s": round(dt_dev, 6), "sources_pro_rata_s": round(src_s, 6),
                   "what": "value = cells x steps / (window device time + sources_ms x steps)"},
        "fp64": {"value": round(value64, 4), "unit": UNIT, "ms_per_step": round((dt64 + src64_s) / args.steps * 1e3, 4),
                 "kernel_ms": kt64},
        "fp32_over_fp64": round(value / value64, 3) if value64 > 0 else None,
        "rel_l2_fp32_vs_fp64": state["diff"] / state["norm"] if state["norm"] > 0 else None,
        "rel_l2_at_step": sim_time_after(t0_window, args),
        "accuracy_4000_steps": accuracy,
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


def sim_time_after(t0_window: int, args) -> int:
    """The time both forms reach after the two timed windows (where
    rel_l2_fp32_vs_fp64 is taken)."""
    return t0_window + args.steps


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
    computes J (mp_objective), of mp_adjoint (forward with checkpoints +
    reverse pass) and of the same in two calls (mp_objective_record, then
    mp_adjoint_reverse), best of three; FP32 and FP64 with a checkpoint every
    50 steps (the workload's schedule) and with the whole E history kept, and
    the FP32 gradient against the FP64 one."""
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
        # the same gradient in two calls: the forward run keeping the
        # checkpoints (mp_objective_record), then the reverse pass
        # (mp_adjoint_reverse), each timed on its own, best of three
        t_rec = t_rev = None
        for _ in range(3):
            with fresh() as g:
                t0 = time.perf_counter()
                g.objective_record(adj)
                t1 = time.perf_counter()
                _, grr = g.adjoint_reverse()
                t2 = time.perf_counter()
            t_rec = t1 - t0 if t_rec is None else min(t_rec, t1 - t0)
            t_rev = t2 - t1 if t_rev is None else min(t_rev, t2 - t1)
        grads[tag] = gr["DesignEps"]
        out[tag] = {"forward_s": round(fwd, 4), "adjoint_s": round(t_adj, 4),
                    "ratio": round(t_adj / fwd, 3), "checkpoint_every": adj.checkpoint_every,
                    "adjoint_full_history_s": round(t_full, 4), "ratio_full_history": round(t_full / fwd, 3),
                    "record_s": round(t_rec, 4), "reverse_s": round(t_rev, 4),
                    "ratio_reverse": round(t_rev / fwd, 3),
                    "ratio_record_plus_reverse": round((t_rec + t_rev) / fwd, 3),
                    "reverse_gradient_equals_adjoint": all(np.array_equal(grr[k], gr[k]) for k in gr),
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
    memory budget of args.budget_gb GB for checkpoints and history and
    args.host_gb GB of pinned host memory for segment checkpoints (the library
    picks the schedule); then the FP32 gradient against the FP64 adjoint on a
    64^3 crop of the workload (16^3 design region, 320 steps)."""
    from mpulse_b200 import runtime
    out = {"adjoint_large_run": True, "steps": args.steps, "budget_gb": args.budget_gb, "host_gb": args.host_gb}
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
        g.set_host_checkpoint_budget(args.host_gb * 1e9)  # pins the host buffers once per context
        out["host_pin_s"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        out["J_adjoint"], gr = g.adjoint(adj)
        out["adjoint_s"] = time.perf_counter() - t0
    out["ratio"] = out["adjoint_s"] / out["forward_s"]
    out["grad_norm_eps"] = float(np.linalg.norm(gr["DesignEps"]))
    if not args.crop:
        return out
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
    """FP32 workload only: pre-roll, warm-up, then the timed steps; no other
    kernels (for ncu captures: the E half's launches are the odd ones from
    launch 2 (args.preroll + args.warmup) on, counting one source batch per 64
    steps)."""
    import torch
    from mpulse_b200 import runtime
    torch.cuda.set_device(0)
    cfg = bench_config(abi.MP_FP32)
    stream = torch.cuda.Stream()
    sim = runtime.Simulation(cfg)
    sim.set_stream(stream.cuda_stream)
    sim.step(args.preroll + args.warmup)
    L0 = sim.launches
    sim.kerr_counts()
    dt, launches = time_steps(sim, torch, args.steps, stream)
    solves, iters = sim.kerr_counts()
    cells = cfg.nx * cfg.ny * cfg.nz
    kt = sim.kernel_times(5)
    sim.close()
    return {"profile_run": True, "grid": [cfg.nx, cfg.ny, cfg.nz], "steps": args.steps, "preroll": args.preroll,
            "launches_before_window": L0, "value": cells * args.steps / dt / 1e9, "unit": UNIT,
            "gpu_launches": launches, "kerr_solves_per_step": solves / args.steps,
            "newton_iterations_per_solve": iters / solves if solves else None, "kernel_ms": kt}


def run_e2e(args, torch, sim, cfg) -> dict:
    """The metric through the C ABI with host buffers, on the simulation's
    current state: mp_upload of the six fields from pinned host memory (the
    state itself, downloaded before the timed region), mp_step(K), mp_download
    of Ex, Ey, Ez, timed by the wall clock."""
    count = cfg.field_count()
    host_in = {n: torch.zeros(count, dtype=torch.float64, pin_memory=True).numpy() for n in abi.FIELD_NAMES}
    host_out = {n: torch.zeros(count, dtype=torch.float64, pin_memory=True).numpy() for n in ("Ex", "Ey", "Ez")}
    for n in abi.FIELD_NAMES:
        sim.download(n, host_in[n])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for n in abi.FIELD_NAMES:
        sim.upload(n, host_in[n])
    sim.step(args.steps)
    for n in ("Ex", "Ey", "Ez"):
        sim.download(n, host_out[n])
    t1 = time.perf_counter()
    cells = cfg.nx * cfg.ny * cfg.nz
    return {"value": round(cells * args.steps / (t1 - t0) / 1e9, 4), "unit": UNIT,
            "h2d_bytes_per_step": int(6 * count * 8 / args.steps), "d2h_bytes_per_step": int(3 * count * 8 / args.steps),
            "what": "mp_upload x6 (pinned double) + mp_step(K) + mp_download x3 on the pre-rolled state, wall clock"}


# ---------------------------------------------------------------------------
# The reference on the host cores.

def _ref_binary():
    for name in ("mpulse_ref_fast", "mpulse_ref"):
        p = os.path.join(ROOT, "oracle", "_ref", name)
        if os.path.exists(p):
            return p
    return None


def reference_state_init(cfg: abi.Config) -> str:
    """pulse_init block (GaussPulseInit, pulseinit.cpp:7-74) of the state the
    reference is timed on: a By/Ex Gaussian pulse with the workload's carrier
    (800 nm), waist (2 um) and length (20 fs FWHM) centred at z = 111, where
    the pre-rolled state of the GPU arm has its peak; as there, the field is
    non-zero in every medium cell, so every cell takes the Kerr solve."""
    k0 = 2 * math.pi / 0.8
    z0 = configs.field_fwhm_to_t0(20.0)  # spatial 1/e half-width c T
    return (f"pulse_init {{ k {k0!r} r0 2.0 z0 {z0!r} zc {111 * cfg.dz!r} C 0 Bx 0 By 1 bound 0 }}")


def reference_slabs(steps: int, warmup: int, procs: int) -> dict:
    """Runs the reference build on the bench workload as `procs` z-slab
    processes, MPulse's own slab decomposition of its MPI build
    (mpi_bound.cpp:66-109) without the halo exchange: each process holds the
    planes of its slab of the one 256 x 256 x 512 grid (the harness's
    slab_xy_periodic boundary), so the CPML z faces, the injection plane and
    the vacuum / medium split sit only in the slabs that contain them and the
    processes together do the whole grid's per-cell work.  Every slab starts
    from reference_state_init, runs warmup + steps steps, and times the last
    `steps`; returns the aggregate rate (all cells over the slowest process's
    time) and the median per-process rate."""
    from oracle import pyoracle
    binary = _ref_binary()
    cfg = bench_config(abi.MP_FP64)
    nz_slab = max(-(-cfg.nz // procs), cfg.cpml_d + 1)  # a slab holds at most one z face
    slabs = [(z, min(z + nz_slab - 1, cfg.nz)) for z in range(1, cfg.nz + 1, nz_slab)]
    tmp = tempfile.mkdtemp(prefix="mpref_bench_")
    init = reference_state_init(cfg)
    runs = []
    for p, (z0, z1) in enumerate(slabs):
        d = os.path.join(tmp, f"r{p}")
        os.makedirs(d)
        with open(os.path.join(d, "setup.dat"), "w") as f:
            f.write(pyoracle.setup_text(cfg, warmup + steps, inits=init,
                                        boundary=f"slab_xy_periodic {{ z0 {z0} z1 {z1} }}"))
        env = dict(os.environ, MPULSE_REF_WARMUP=str(warmup))
        runs.append(subprocess.Popen([binary, os.path.join(d, "setup.dat"), d], stdout=subprocess.PIPE,
                                     stderr=subprocess.DEVNULL, env=env, text=True))
    secs, cells, rates = [], 0, []
    for pr in runs:
        outp, _ = pr.communicate()
        if pr.returncode != 0:
            raise RuntimeError("reference run failed")
        r = json.loads(outp.strip().splitlines()[-1])
        secs.append(r["seconds"])
        cells += r["cells"]
        rates.append(r["cells"] * steps / r["seconds"] / 1e9)
    t = max(secs)
    return {"value": cells * steps / t / 1e9, "procs": len(slabs), "cells": cells, "seconds": t,
            "nz_slab": nz_slab, "per_core": float(np.median(rates))}


def _reference_sample_text(r: dict, warmup: int, steps: int) -> str:
    return (f"MPulse reference build (-O3), the one 256x256x512 grid of the workload as {r['procs']} z-slab processes "
            f"of {r['nz_slab']} planes (MPulse's MPI slab split without the halo exchange; CPML faces and "
            f"injection plane only where the grid has them), from a pulse_init state in the Kerr medium, "
            f"{warmup} warm-up + {steps} timed steps")


def cpu_baseline_sample(args) -> dict:
    """Bounded CPU baseline for the headline line: the reference build on the
    host cores for 2 timed steps of the full workload, as z-slabs."""
    if _ref_binary() is None:
        return cpu_baseline_port()
    procs = max(1, min(os.cpu_count() or 1, 64))
    r = reference_slabs(steps=2, warmup=1, procs=procs)
    return {"value": round(r["value"], 6), "unit": UNIT, "cores": r["procs"], "kind": "reference",
            "sample": _reference_sample_text(r, 1, 2), "same_config": True,
            "per_core_value": round(r["per_core"], 6),
            "per_core": "median rate of one slab process (the reference is single-threaded), measured while all ran"}


def cpu_baseline_port() -> dict:
    from oracle import pyoracle
    c = bench_config(abi.MP_FP64)
    c.nz = 32
    c.medium_z0 = 0
    o = pyoracle.OracleSim(c)
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
    cfg = bench_config(abi.MP_FP64)
    return {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": 0, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(r["seconds"] / args.steps * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config_keys(cfg),
        "parallelism": f"{r['procs']} processes",
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": r["procs"], "kind": "reference",
                         "sample": _reference_sample_text(r, args.warmup, args.steps), "same_config": True,
                         "per_core_value": round(r["per_core"], 6)},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": round(wall, 2),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--preroll", type=int, default=PREROLL_STEPS,
                    help="untimed steps from time 0 before the warm-up (pulse into the Kerr medium)")
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--profile-only", action="store_true",
                    help="only the FP32 warm-up and timed steps (for ncu captures)")
    ap.add_argument("--nz", type=int, default=None, help="override nz (smaller case for ncu --set full)")
    ap.add_argument("--adjoint-only", action="store_true",
                    help="only mp_objective + mp_adjoint of the adjoint workload for --steps steps (ncu captures)")
    ap.add_argument("--checkpoint", type=int, default=50, help="checkpoint interval of --adjoint-only")
    ap.add_argument("--adjoint-ratio", action="store_true",
                    help="only the adjoint workload's wall-time ratios (the `adjoint` object of the bench line)")
    ap.add_argument("--adjoint-large", action="store_true",
                    help="the 512x512x768 nonlinear adjoint workload for --steps steps (minutes)")
    ap.add_argument("--budget-gb", type=float, default=120.0, help="checkpoint budget of --adjoint-large")
    ap.add_argument("--host-gb", type=float, default=0.0,
                    help="pinned host memory for the segment checkpoints of --adjoint-large")
    ap.add_argument("--no-crop", dest="crop", action="store_false", help="--adjoint-large without the 64^3 crop")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.nz:
        WORKLOAD["nz"] = args.nz
    if args.adjoint_ratio:
        out = run_adjoint(0)
    elif args.adjoint_large:
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
