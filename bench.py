#!/usr/bin/env python
"""Throughput of the fused Model C step on B200 (Gcell-updates/s).

Workload (default, --config c3): Karma-Rappel Model C on 10080^2 =
101,606,400 cells as 80x80 blocks of 126^2, ghost 1, h = 0.4, dt = 0.008,
D = 2, lambda = D/0.6267, eps4 = 0.05, u0 = -0.5, 64 seeded grains of radius
8, zero-flux boundaries, Gaussian noise b = 0.01, Euler-Maruyama, FP64.  A
step is one time step over the whole grid (101.6M cell-updates).  The state
(2 fields x 2 buffers, 4.2 GB) is far larger than L2, so no flush is needed
between steps.  --config c2 is the 4096^2 grid of 16x16 blocks of 256^2.

Arms:
  default          this library on N GPUs (N independent replicas, one per
                   rank, weak scaling; the path has no cross-replica exchange)
  --impl reference the reference's CPU path (the oracle restatement, all host
                   threads) on rank 0, same config and metric.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

CONFIGS = {
    # Model C 2D, 4096^2 as 16x16 blocks of 256^2
    "c2": dict(workload="model_c_4096sq", cells=4096, block=256, h=0.4, dt=0.008, d_thermal=2.0,
               lam=2.0 / 0.6267, eps4=0.05, u0=0.55, grains=16, radius=8.0, noise=0.01, seed=42,
               full_steps=20000),
    # Model C 2D at full scale, 10080^2 as 80x80 blocks of 126^2
    "c3": dict(workload="model_c_10080sq", cells=10080, block=126, h=0.4, dt=0.008, d_thermal=2.0,
               lam=2.0 / 0.6267, eps4=0.05, u0=0.5, grains=64, radius=8.0, noise=0.01, seed=42,
               full_steps=10000),
    # the reference's flagship run (README: model_c --cells 10080 --block 126
    # --seeds 1000 --orient --noise 0.02): classic Model C (eps4 0.06, lambda
    # 3.19, D = 0.6267 lambda), 1000 grains of r = 10 h with orientations
    # unit_open(mix_key(42, [i, 2])) pi/2, theta0 by nearest seed, u0 = 0.7,
    # b = 0.02, dt = 0.2 h^2 / D
    "c3o": dict(workload="model_c_10080sq_1000grains_oriented", cells=10080, block=126, h=0.4,
                dt=0.2 * 0.4 * 0.4 / (0.6267 * 3.19), d_thermal=0.6267 * 3.19, lam=3.19, eps4=0.06, u0=0.7,
                grains=1000, radius=4.0, noise=0.02, seed=42, orient=True, full_steps=21865),
    # 3-D heat, 96^3 periodic as 6^3 blocks of 16^3, dt = 0.15 h^2, sine + seeded noise
    "c1": dict(kind="heat", workload="heat_96cube", cells=96, block=16, kappa=1.0, seed=42, amp=1e-3,
               full_steps=2000, noise=0.0),
    # the same heat model at 512^3 (32^3 blocks of 16^3): an HBM-resident variant
    "c1big": dict(kind="heat", workload="heat_512cube", cells=512, block=16, kappa=1.0, seed=42, amp=1e-3,
                  full_steps=2000, noise=0.0),
    # Model C with Berger-Oliger AMR: 1024^2 base as 32^2 blocks of 32^2,
    # ratios [2, 2, 2], tag |grad phi| > 0.05, regrid every 50 coarse steps,
    # one central grain r = 8, u0 = -0.55, no noise, subcycled
    "c4": dict(kind="amr", workload="model_c_amr_1024sq_3lev", cells=1024, block=32, h=0.4, d_thermal=2.0,
               lam=2.0 / 0.6267, eps4=0.05, u0=0.55, radius=8.0, ratios=[2, 2, 2], every=50, buffer=2,
               threshold=0.05, noise=0.0, full_steps=4000),
    # batched ensemble + adjoint: 256 instances of 256^2 as 4x4 blocks of 64^2,
    # per-instance eps4 ~ U[0.02, 0.07], Delta ~ U[0.45, 0.65] and seed drawn
    # by unit_open(mix_key(master, [i, k])); one central grain r = 8; noise
    # b = 0.005; FP32 forward, FP64 gradient accumulation; 2000 steps with a
    # checkpoint every 100; loss against phi_T at perturbed eps4 and Delta
    "c5": dict(kind="ensemble", workload="model_c_ensemble_256x256sq", instances=256, cells=256, block=64, h=0.4,
               d_thermal=2.0, lam=2.0 / 0.6267, radius=8.0, noise=0.005, seed=42, ckpt=100, full_steps=2000),
}

BYTES_PER_CELL = {"f64": 32, "f32": 16}  # read phi, u; write phi, u

# DRAM bytes (read + write) per cell-update of the dominant kernel, from one
# ncu capture each of the kernel as it now is (the summaries under
# profiles/ named in NCU_INST): the FP64 and FP32 strip kernels in the
# variant the autotuner picks on 10080^2 (CAPTURED_VARIANT), captured on
# 5040^2 of the same 126^2 blocks (833.3 MB and 375.4 MB per 25.4M-cell
# launch), and the TMA-staged 3-D heat kernel on 256^3 (319.7 MB per 16.8M
# cells; 512^3 has the same per-block work).  Traffic grows with the cell
# count, so a launch of the full grid moves the per-cell figure times its
# cells.  Other workloads report null.
TRAFFIC_PER_CELL = {("c3", "f64"): 827.2e6 / 5040 ** 2, ("c3", "f32"): 377.0e6 / 5040 ** 2,
                    ("c1big", "f64"): 274.3e6 / 256 ** 3}

NOMINAL_HBM_GBS = 8000.0  # a B200's nominal HBM3e bandwidth, the second denominator

# Instruction mix of the dominant kernel per cell-update, from the same
# captures (smsp__inst_executed and the fp64 pipe's share, x 32 threads per
# warp instruction, divided by the launch's cell-updates); the capture named
# is the summary under profiles/.
NCU_INST = {("c3", "f64"): {"inst_per_cell": 408.7, "fp64_inst_per_cell": 126.8,
                            "capture": "modelc_strip_f64_5040sq_126blocks"},
            ("c3", "f32"): {"inst_per_cell": 242.4, "fp64_inst_per_cell": None,
                            "capture": "modelc_strip_f32_5040sq_126blocks"},
            ("c1big", "f64"): {"inst_per_cell": 73.3, "fp64_inst_per_cell": None,
                               "capture": "heat3d_tma_256cube"}}

# the strip-kernel variant the captures ran (the autotuner's choice on 10080^2)
CAPTURED_VARIANT = 32015


def compute_roofline(peaks, sm_mhz, cells_per_s, ncu):
    """The compute side of the roofline: the kernel's thread-instruction rate
    against the issue ceiling (one warp instruction per SM sub-partition per
    clock at the sampled SM clock) and its FP64 operation rate against the
    measured FP64 FMA rate of the device (lg_measure_compute_peaks)."""
    if peaks is None:
        return None
    clock = sm_mhz if sm_mhz else peaks["clock_mhz"]
    issue_ceiling = peaks["sms"] * 4 * 32 * clock * 1e6
    out = {"issue_ceiling_thread_inst_per_s": issue_ceiling, "clock_mhz": clock,
           "measured": {k: peaks[k] for k in ("dfma_per_s", "ffma_per_s", "imad_per_s", "alu_per_s")},
           "inst_per_cell": None, "issue_frac": None, "fp64_inst_per_cell": None, "fp64_frac": None,
           "capture": None}
    if ncu:
        out["capture"] = ncu["capture"]
        out["inst_per_cell"] = ncu["inst_per_cell"]
        out["issue_frac"] = ncu["inst_per_cell"] * cells_per_s / issue_ceiling
        if ncu.get("fp64_inst_per_cell") is not None:
            out["fp64_inst_per_cell"] = ncu["fp64_inst_per_cell"]
            out["fp64_frac"] = ncu["fp64_inst_per_cell"] * cells_per_s / peaks["dfma_per_s"]
    return out


def ncu_capture_config(args) -> bool:
    """True when the run is the configuration the ncu figures were taken on:
    no size, noise, integrator or kernel-variant override (variant 0 runs the
    autotuner's choice, which on the captured grids is CAPTURED_VARIANT)."""
    return (args.cells is None and args.noise is None and args.integrator == "em"
            and args.variant in (0, CAPTURED_VARIANT))


def traffic(args, cells_per_step):
    """Measured DRAM bytes per launch of the dominant kernel, or None."""
    if not ncu_capture_config(args):
        return None
    per = TRAFFIC_PER_CELL.get((args.config, args.dtype))
    return None if per is None else per * cells_per_step


def hbm_roofline(achieved, peak, peak_kind, **more):
    """The roofline object: achieved GB/s against the measured copy bandwidth
    (or the fallback) and against the nominal 8 TB/s."""
    r = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
         "peak_kind": peak_kind, "nominal_peak": NOMINAL_HBM_GBS, "frac_nominal": achieved / NOMINAL_HBM_GBS}
    r.update(more)
    return r


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi sampled every 200 ms while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-f", self.path], stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in Path(self.path).read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup(n_gpus: int):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch

    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist
    return rank, world, local, pg


def barrier(pg):
    if pg is not None:
        pg.barrier()


def max_over_ranks(pg, value: float) -> float:
    if pg is None:
        return value
    import torch

    # NCCL reduces device tensors; gloo (the host-side tests) host ones
    t = torch.tensor([value], dtype=torch.float64, device="cuda" if pg.get_backend() == "nccl" else "cpu")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def make_sim(cfg, dtype, sched, seed_offset=0):
    import legendre_b200 as L

    n, b, h = cfg["cells"], cfg["block"], cfg["h"]
    grid = L.CartesianGrid([n, n], [b, b], [0.0, 0.0], [h, h])
    model = L.ModelC(cfg["eps4"], cfg["lam"], cfg["noise"])
    model.d_thermal = cfg["d_thermal"]
    if cfg.get("orient"):
        model.with_orientations()
    integrator = L.RungeKutta4() if cfg.get("integrator") == "rk4" else L.EulerMaruyama(cfg["seed"] + seed_offset)
    sim = L.Simulation(grid, L.FiniteVolume(), model, integrator, sched, L.CudaAllocator(dtype))
    grains = L.seed_positions(n, h, cfg["grains"], cfg["seed"], radius=cfg["radius"], orient=cfg.get("orient", False))
    return sim, grid, model, grains


def initialize(sim, grid, model, grains, cfg, dtype, sched):
    import numpy as np

    import legendre_b200 as L

    if dtype == "f64":
        model.initialize_grains(grid, sim.state, grains, cfg["u0"])
        return
    tmp = L.DeviceState(grid, sched, L.CudaAllocator("f64"), sim.state.specs)
    model.initialize_grains(grid, tmp, grains, cfg["u0"])
    for spec in sim.state.specs:
        sim.state.upload(spec.name, tmp.download(spec.name).astype(np.float32))
    tmp._destroy()
    if model.orientations:
        model.set_orientations(sim.state)


def to_global(blocks, n, b):
    """(num_blocks, b, b) block-major interiors -> (n, n), row-major."""
    nb = n // b
    return blocks.reshape(nb, nb, b, b).transpose(0, 2, 1, 3).reshape(n, n)


def tip_position(phi, row, x0, h):
    """x of the last zero crossing of phi along `row` to the right of x0
    (linear interpolation between cell centres): the +x dendrite tip."""
    line = phi[row]
    i = int(x0 / h)
    while i + 1 < line.size and line[i + 1] > 0.0:
        i += 1
    if i + 1 >= line.size or line[i] <= 0.0:
        return float("nan")
    return ((i + 0.5) + line[i] / (line[i] - line[i + 1])) * h


TIP_DIRECTIONS = ((1, 0), (-1, 0), (0, 1), (0, -1))  # +x, -x, +y, -y


def tip_extents(phi, centers, h):
    """Distance from each grain centre to the phi = 0 crossing along +x, -x,
    +y and -y: walk from the centre's cell while phi > 0, then interpolate
    linearly between the last solid cell centre and the next one.  nan
    where the centre is not solid or the walk leaves the domain.  phi is
    (rows = y, columns = x); returns (len(centers), 4)."""
    import numpy as np

    ny, nx = phi.shape
    out = np.full((len(centers), len(TIP_DIRECTIONS)), np.nan)
    for g, (cx, cy) in enumerate(centers):
        i0, j0 = int(cx / h), int(cy / h)
        if not (0 <= i0 < nx and 0 <= j0 < ny) or phi[j0, i0] <= 0.0:
            continue
        for k, (di, dj) in enumerate(TIP_DIRECTIONS):
            i, j = i0, j0
            while 0 <= i + di < nx and 0 <= j + dj < ny and phi[j + dj, i + di] > 0.0:
                i, j = i + di, j + dj
            if not (0 <= i + di < nx and 0 <= j + dj < ny):
                continue
            a, b = phi[j, i], phi[j + dj, i + di]
            frac = a / (a - b)
            x, y = (i + 0.5 + di * frac) * h, (j + 0.5 + dj * frac) * h
            out[g, k] = abs(x - cx) if di else abs(y - cy)
    return out


def fp32_error(cfg, sched, steps):
    """The FP32 path against the FP64 path (bit-identical to the CPU
    oracle) from the same initial state and noise keys: phi L2 (RMS) and
    L-inf after `steps` steps, solid fractions (phi > 0), the tip velocities
    over the second half (the phi = 0 crossings along +-x and +-y of every
    grain; the +x tip of the grain nearest the domain centre separately),
    and the total enthalpy h^2 sum(u - phi/2) at the start and the end (FP64
    device sums; the noise moves it, the deterministic step only by
    rounding)."""
    import numpy as np

    n, b, h = cfg["cells"], cfg["block"], cfg["h"]
    out = {}
    for dtype in ("f64", "f32"):
        sim, grid, model, grains = make_sim(cfg, dtype, sched)
        initialize(sim, grid, model, grains, cfg, dtype, sched)
        h0 = model.enthalpy(grid, sim.state)
        c = min(grains, key=lambda g: (g.center[0] - n * h / 2) ** 2 + (g.center[1] - n * h / 2) ** 2)
        row = int(c.center[1] / h)
        sim.run(cfg["dt"], steps // 2, graph=True)
        p1 = to_global(sim.state.interior("phi").astype(np.float64), n, b)
        sim.run(cfg["dt"], steps - steps // 2, graph=True)
        p2 = to_global(sim.state.interior("phi").astype(np.float64), n, b)
        span = (steps - steps // 2) * cfg["dt"]
        v = (tip_position(p2, row, c.center[0], h) - tip_position(p1, row, c.center[0], h)) / span
        centers = [gr.center for gr in grains]
        v_all = (tip_extents(p2, centers, h) - tip_extents(p1, centers, h)) / span
        out[dtype] = (p2, v, float(np.mean(p2 > 0.0)), (h0, model.enthalpy(grid, sim.state)), v_all)
        del sim
    d = out["f32"][0] - out["f64"][0]
    v64, v32 = out["f64"][4], out["f32"][4]
    ok = np.isfinite(v64) & np.isfinite(v32) & (np.abs(v64) > 1e-12)
    tip_rel = np.abs(v32[ok] - v64[ok]) / np.abs(v64[ok])
    return {"steps": steps, "phi_l2": float(np.sqrt(np.mean(d * d))), "phi_linf": float(np.max(np.abs(d))),
            "solid_fraction_f64": out["f64"][2], "solid_fraction_f32": out["f32"][2],
            "tip_velocity_f64": out["f64"][1], "tip_velocity_f32": out["f32"][1],
            "tip_velocity_rel_err": abs(out["f32"][1] - out["f64"][1]) / abs(out["f64"][1]),
            "tips": int(ok.sum()), "tip_velocity_mean_f64": float(np.mean(v64[ok])) if ok.any() else None,
            "tip_velocity_max_rel_err": float(np.max(tip_rel)) if ok.any() else None,
            "tip_velocity_median_rel_err": float(np.median(tip_rel)) if ok.any() else None,
            "enthalpy_f64": list(out["f64"][3]), "enthalpy_f32": list(out["f32"][3]),
            "enthalpy_rel_diff": abs(out["f32"][3][1] - out["f64"][3][1]) / abs(out["f64"][3][1]),
            "reference": "the FP64 device path from the same state and noise keys: bit-identical to the CPU "
                         "oracle without noise and within 1e-12 of it with noise (the GPU tests check both, and "
                         "FP32 against the oracle itself at 4096^2)"}


def cpu_oracle_rate(cfg, steps_budget_s: float, max_steps: int, warmup: int = 1):
    """Oracle (C++ restatement of the reference's CPU path), all host threads,
    on the full grid; returns (Gcell/s, steps run, threads, ms per step).
    Loads only the oracle's library: the seed placement comes from the
    package's pure-Python module, which maps no device code."""
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_bind as orc

    from legendre_b200.seeding import seed_positions

    n, b, h = cfg["cells"], cfg["block"], cfg["h"]
    og = orc.Grid([n, n], [b, b], [0.0, 0.0], [h, h])
    orient = bool(cfg.get("orient"))
    st = orc.State(og, [1, 1, 0] if orient else [1, 1])
    grains = seed_positions(n, h, cfg["grains"], cfg["seed"], radius=cfg["radius"], orient=orient)
    st.initialize_grains([(g.center[0], g.center[1], g.radius) for g in grains], cfg["u0"])
    if orient:
        st.initialize_orientations(2, [(g.center[0], g.center[1], g.radius, g.orientation) for g in grains])
    p = orc.modelc_params(eps4=cfg["eps4"], lam=cfg["lam"], d_thermal=cfg["d_thermal"], noise=cfg["noise"])
    threads = int(orc.lib.orc_num_threads_available())

    def run(t, k):
        if orient:
            return st.modelc_run_oriented(p, 2, t, cfg["dt"], cfg["seed"], k, True, threads)
        return st.modelc_run(p, t, cfg["dt"], cfg["seed"], k, True, threads)

    t0 = time.perf_counter()
    t = run(0.0, max(1, warmup))
    one = (time.perf_counter() - t0) / max(1, warmup)
    steps = max(1, min(max_steps, int(steps_budget_s / max(one, 1e-6))))
    t0 = time.perf_counter()
    run(t, steps)
    el = time.perf_counter() - t0
    return n * n * steps / el / 1e9, steps, threads, 1e3 * el / steps


def run_reference(args, cfg):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    rate, steps, threads, ms_step = cpu_oracle_rate(cfg, steps_budget_s=60.0, max_steps=args.steps,
                                                    warmup=args.warmup)
    line = {
        "metric": "Gcell-updates/s", "value": rate, "unit": "Gcell-updates/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": cfg["workload"], "cells": cfg["cells"], "block": cfg["block"], "noise": cfg["noise"]},
        "cpu_baseline": {"value": rate, "unit": "Gcell-updates/s", "cores": threads, "kind": "port",
                         "sample": f"{steps} of {args.steps} steps on the full {cfg['cells']}^2 grid "
                                   f"(after {args.warmup} warm-up steps)"},
        "e2e": {"value": rate, "unit": "Gcell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference (Rust) cannot be built here; this arm times the C++ restatement of its "
                "SerialScheduler path with OpenMP over blocks (RayonScheduler's parallelism)",
    }
    print(json.dumps(line), flush=True)


def run_other(args, cfg):
    """The heat (c1) and AMR (c4) configurations: device-timed K steps,
    the same JSON schema (no CPU leg, no e2e copy-in/out)."""
    import math

    import numpy as np
    import torch

    import legendre_b200 as L

    rank, world, local, pg = dist_setup(args.gpus)
    stream = torch.cuda.Stream(device=local)
    torch.cuda.set_stream(stream)
    sched = L.CudaScheduler(local, stream.cuda_stream)
    if cfg["kind"] == "heat":
        n, b = cfg["cells"], cfg["block"]
        h = 1.0 / n
        grid = L.CartesianGrid([n] * 3, [b] * 3, [0.0] * 3, [h] * 3).with_periodic([True] * 3)
        model = L.Heat(cfg["kappa"])
        sim = L.Simulation(grid, L.FiniteDifference(), model, L.ForwardEuler(), sched, L.CudaAllocator("f64"))
        model.initialize_sine_noise(sim.state, cfg["seed"], cfg["amp"])
        dt = 0.15 * h * h
        run = lambda k: sim.run(dt, k, graph=True)
        cells_per_step = lambda: float(n ** 3)
        bytes_per_cell = 16
        extra = {"cells": n, "block": b, "periodic": True, "dt": dt,
                 "l2": "state fits in L2 (no flush): launch- and L2-bound" if n ** 3 * 8 * 2 < 100e6
                 else "state larger than L2; no flush"}
    else:
        n, b, hh = cfg["cells"], cfg["block"], cfg["h"]
        base = L.CartesianGrid([n, n], [b, b], [0.0, 0.0], [hh, hh])
        grid = L.AmrGrid.from_patches(base, cfg["ratios"], [])
        model = L.ModelC(cfg["eps4"], cfg["lam"], cfg["noise"])
        model.d_thermal = cfg["d_thermal"]
        adapt = L.BergerOliger(L.GradientTagger("phi", cfg["threshold"]),
                               L.RegridPolicy(cfg["every"], cfg["buffer"], L.ClusterParams(0.8, 4)))
        sim = L.AmrSimulation(grid, L.FiniteVolume(), model, L.Subcycling(0), sched, L.CudaAllocator("f64"), adapt)
        c = n * hh / 2.0
        phi, u = sim.get("phi"), sim.get("u")
        for k in range(sim.num_blocks):
            xs, ys = sim.centers(k)
            r = np.hypot(xs - c, ys - c)
            phi[k][1:-1, 1:-1] = np.maximum(-1.0, -np.tanh((r - cfg["radius"]) / math.sqrt(2.0)))
            u[k][1:-1, 1:-1] = -cfg["u0"]
        sim.set("phi", phi)
        sim.set("u", u)
        dt = sim.stable_dt()
        run = lambda k: sim.run(dt, k, graph=True)

        def cells_per_step():
            # cell-updates of one coarse step: every level's cells times its
            # substeps per coarse step (4 per level at ratio 2)
            tot, mult = 0.0, 1.0
            per_level = {}
            for lv, lo, hi in sim.patches():
                per_level[lv] = per_level.get(lv, 0) + (hi[0] - lo[0]) * (hi[1] - lo[1])
            for lv in sorted(per_level):
                tot += per_level[lv] * mult
                mult *= 4.0
            return tot
        bytes_per_cell = 32
        extra = {"cells": n, "block": b, "ratios": cfg["ratios"], "regrid_every": cfg["every"], "dt": dt,
                 "l2": "hierarchy state below L2 size; no flush"}
    run(args.warmup)
    torch.cuda.synchronize()
    c0 = cells_per_step()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    barrier(pg)
    torch.cuda.synchronize()
    launches0 = sched.kernel_launches
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    run(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    launches = sched.kernel_launches - launches0
    barrier(pg)
    clk = clocks.stop()
    c1 = cells_per_step()
    ms = max_over_ranks(pg, e0.elapsed_time(e1))
    cells = 0.5 * (c0 + c1)
    value = world * cells * args.steps / (ms / 1e3) / 1e9
    if rank == 0:
        peak, peak_kind = peaks()
        achieved = bytes_per_cell * cells / (ms / args.steps / 1e3) / 1e9
        line = {
            "metric": "Gcell-updates/s", "value": value, "unit": "Gcell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict({"workload": cfg["workload"], "parallelism": f"replicas{world}", "graph": True}, **extra),
            "roofline": hbm_roofline(achieved, peak, peak_kind,
                                     traffic=traffic(args, cells) if cfg["kind"] == "heat" else None,
                                     algorithmic_bytes_per_cell=bytes_per_cell,
                                     compute=compute_roofline(sched.compute_peaks(), clk.get("sm_mhz"),
                                                              value * 1e9 / world,
                                                              NCU_INST.get((args.config, "f64"))
                                                              if ncu_capture_config(args) else None)),
            "cpu_baseline": None, "e2e": None,
            "gpu_launches": launches,
            "clocks": {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"],
                       "samples": clk["samples"]},
        }
        print(json.dumps(line), flush=True)
    sched.close()
    if pg is not None:
        pg.destroy_process_group()


def ensemble_setup(cfg, ninst):
    """Per-instance eps4, Delta, seed and the initial fields of the ensemble
    workload (instances, ny, nx)."""
    import math

    import numpy as np

    from legendre_b200.rng import mix_key, unit_open

    m = cfg["seed"]
    eps4 = [0.02 + 0.05 * unit_open(mix_key(m, [i, 0])) for i in range(ninst)]
    delta = [0.45 + 0.2 * unit_open(mix_key(m, [i, 1])) for i in range(ninst)]
    seeds = [mix_key(m, [i, 2]) for i in range(ninst)]
    n, h = cfg["cells"], cfg["h"]
    x = (np.arange(n) + 0.5) * h
    r = np.hypot(x[None, :] - n * h / 2, x[:, None] - n * h / 2)
    phi = np.maximum(-1.0, -np.tanh((r - cfg["radius"]) / math.sqrt(2.0)))
    phi0 = np.broadcast_to(phi, (ninst, n, n))
    u0 = -np.asarray(delta)[:, None, None] * np.ones((1, n, n))
    return eps4, delta, seeds, phi0, u0


def run_ensemble(args, cfg):
    """The batched ensemble (c5): forward throughput of all instances, and
    the cost of the value-and-gradient pass against the forward pass alone."""
    import numpy as np
    import torch

    import legendre_b200 as L

    rank, world, local, pg = dist_setup(args.gpus)
    stream = torch.cuda.Stream(device=local)
    torch.cuda.set_stream(stream)
    sched = L.CudaScheduler(local, stream.cuda_stream)
    dtype = args.dtype if args.dtype_given else "f32"
    ninst, n, b, h = cfg["instances"], cfg["cells"], cfg["block"], cfg["h"]
    grid = L.CartesianGrid([n, n], [b, b], [0.0, 0.0], [h, h])
    model = L.ModelC(0.05, cfg["lam"], cfg["noise"])
    model.d_thermal = cfg["d_thermal"]
    eps4, delta, seeds, phi0, u0 = ensemble_setup(cfg, ninst)
    seeds = [(s + rank) % (1 << 64) for s in seeds]
    dt = 0.2 * h * h / cfg["d_thermal"]
    cells = ninst * n * n

    def fresh(e4, dl):
        ens = L.Ensemble(grid, model, e4, seeds, sched, dtype=dtype)
        ens.set("phi", phi0)
        ens.set("u", -np.asarray(dl)[:, None, None] * np.ones((1, n, n)))
        return ens

    # forward throughput
    ens = fresh(eps4, delta)
    ens.run(dt, args.warmup, graph=True)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    barrier(pg)
    torch.cuda.synchronize()
    launches0 = sched.kernel_launches
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ens.run(dt, args.steps, graph=True)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(pg)
    clk = clocks.stop()
    launches = sched.kernel_launches - launches0
    ms = max_over_ranks(pg, e0.elapsed_time(e1))
    value = world * cells * args.steps / (ms / 1e3) / 1e9

    # end to end through the public API: host fields in, K steps, phi out
    barrier(pg)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    ens.set("phi", phi0)
    ens.set("u", u0)
    ens.run(dt, args.steps, graph=True)
    phi_out = ens.get("phi")
    e3.record(stream)
    torch.cuda.synchronize()
    ms_e2e = max_over_ranks(pg, 1e3 * (time.perf_counter() - t0))
    ens._destroy()

    # value and gradient over the configuration's horizon (its full 2000
    # steps, whatever --steps says) against a target at perturbed eps4 and
    # Delta, and the forward pass of the same horizon
    T = cfg["full_steps"]
    tgt = fresh([e + 0.005 for e in eps4], [d + 0.01 for d in delta])
    tgt.run(dt, T, graph=True)
    target = tgt.get("phi")
    tgt._destroy()
    ens = fresh(eps4, delta)
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    ens.run(dt, T, graph=True)
    f1.record(stream)
    torch.cuda.synchronize()
    ms_fwd = f0.elapsed_time(f1)
    ens._destroy()
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed_vg(budget):
        # one untimed pass allocates the workspace (checkpoints, recompute
        # buffers, resident states); the timed pass from the same initial
        # state reuses it
        ens = fresh(eps4, delta)
        ens.value_and_grad(dt, T, cfg["ckpt"], target, cell_grads=False, resident_bytes=budget)
        ens.set("phi", phi0)
        ens.set("u", -np.asarray(delta)[:, None, None] * np.ones((1, n, n)))
        ens.set_time(0.0, 0)
        torch.cuda.synchronize()
        g0.record(stream)
        g = ens.value_and_grad(dt, T, cfg["ckpt"], target, cell_grads=False, resident_bytes=budget)
        g1.record(stream)
        torch.cuda.synchronize()
        ms = g0.elapsed_time(g1)
        ens._destroy()
        return g, ms

    g, ms_vg = timed_vg(0)
    # the same with a resident tail: the last segments that fit in the free
    # device memory (less an 8 GB margin) keep their states from the forward
    # pass instead of being recomputed; the results are the same bits
    free_b, _ = torch.cuda.mem_get_info()
    budget = max(0, int(free_b) - (8 << 30))
    g_res, ms_vg_res = timed_vg(budget)
    same_bits = all(np.array_equal(g[k], g_res[k]) for k in ("loss", "lambda", "d_thermal", "eps4", "delta"))
    state_bytes = ninst * (n // b) ** 2 * 2 * (b + 2) ** 2 * (8 if dtype == "f64" else 4)
    ms_fwd, ms_vg, ms_vg_res = (max_over_ranks(pg, v) for v in (ms_fwd, ms_vg, ms_vg_res))

    if rank == 0:
        peak, peak_kind = peaks()
        bpc = BYTES_PER_CELL[dtype]
        achieved = bpc * cells / (ms / args.steps / 1e3) / 1e9
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            c2 = dict(CONFIGS["c2"], cells=n, block=b, grains=1, noise=cfg["noise"], u0=delta[0], eps4=eps4[0],
                      dt=dt)
            rate, steps_run, threads, _ = cpu_oracle_rate(c2, steps_budget_s=15.0, max_steps=2000)
            cpu = {"value": rate, "unit": "Gcell-updates/s", "cores": threads, "kind": "port",
                   "sample": f"{steps_run} steps of one {n}^2 instance (the instances are independent; the rate "
                             "per cell-update is the same), OpenMP over blocks"}
        esz = 8 if dtype == "f64" else 4
        line = {
            "metric": "Gcell-updates/s", "value": value, "unit": "Gcell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": dtype, "data": "synthetic",
            "config": {"workload": cfg["workload"], "instances": ninst, "cells": n, "block": b,
                       "noise": cfg["noise"], "parallelism": f"replicas{world}", "graph": True,
                       "l2": "state larger than L2; no flush"},
            "roofline": hbm_roofline(achieved, peak, peak_kind, traffic=None, algorithmic_bytes_per_cell=bpc),
            "adjoint": {"steps": T, "checkpoint_every": cfg["ckpt"], "forward_ms": ms_fwd,
                        "value_and_grad_ms": ms_vg, "cost_ratio": ms_vg / ms_fwd,
                        "what": "value_and_grad = forward with checkpoints + loss + per segment: recompute and "
                                "adjoint steps; cost_ratio = its time / the forward pass alone",
                        "mean_loss": float(np.mean(g["loss"])),
                        "mean_grad": {k: float(np.mean(g[k])) for k in ("lambda", "d_thermal", "eps4", "delta")},
                        "resident_tail": {"budget_bytes": budget, "states_fitting": budget // state_bytes,
                                          "value_and_grad_ms": ms_vg_res, "cost_ratio": ms_vg_res / ms_fwd,
                                          "same_bits": same_bits}},
            "cpu_baseline": cpu,
            "e2e": {"value": world * cells * args.steps / (ms_e2e / 1e3) / 1e9, "unit": "Gcell-updates/s",
                    "h2d_bytes_per_step": 2 * cells * 8 / args.steps, "d2h_bytes_per_step": cells * 8 / args.steps,
                    "what": f"Ensemble.set phi and u from host + {args.steps} steps + Ensemble.get phi, "
                            "host wall clock, bytes amortised per step"},
            "gpu_launches": launches,
            "clocks": {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"],
                       "samples": clk["samples"]},
        }
        print(json.dumps(line), flush=True)
    sched.close()
    if pg is not None:
        pg.destroy_process_group()


def model_c_line(args, cfg, world, ms, clk, launches, tuned, e2e, observed, err, cpu, peak, peak_kind,
                 compute_peaks=None):
    """The JSON line of a uniform-grid Model C run from its measured parts
    (device time of the K timed steps `ms`, sampled clocks, launch count,
    autotuner choice, end-to-end and observer blocks, FP32 error, CPU
    baseline and the HBM peak); pure, so it is tested on the host."""
    cells = cfg["cells"] ** 2
    ms_per_step = ms / args.steps
    value = world * cells * args.steps / (ms / 1e3) / 1e9
    # the multi-grain step also reads cos and sin theta0 of every cell; an
    # RK4 step is four stages: three read their input and y and write k and
    # the next input (phi and u of each: 8 values), the last reads its input,
    # y and k1..k3 and writes y (12 values): 36 values per cell
    esz = 8 if args.dtype == "f64" else 4
    bpc = BYTES_PER_CELL[args.dtype] + (2 * esz if cfg.get("orient") else 0)
    if cfg.get("integrator") == "rk4":
        bpc = 36 * esz + (4 * 2 * esz if cfg.get("orient") else 0)
    achieved = bpc * cells / (ms_per_step / 1e3) / 1e9
    captured_cfg = ncu_capture_config(args)
    return {
        "metric": "Gcell-updates/s", "value": value, "unit": "Gcell-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": args.dtype, "data": "synthetic",
        "config": {"workload": cfg["workload"], "cells": cfg["cells"], "block": cfg["block"],
                   "noise": cfg["noise"], "parallelism": f"replicas{world}",
                   "l2": "state 2 fields x 2 buffers larger than L2; no flush",
                   "graph": True, "variant": args.variant, "autotuned_variant": tuned},
        "roofline": hbm_roofline(achieved, peak, peak_kind, traffic=traffic(args, cells),
                                 algorithmic_bytes_per_cell=bpc,
                                 compute=compute_roofline(compute_peaks, clk.get("sm_mhz"), value * 1e9 / world,
                                                          NCU_INST.get((args.config, args.dtype))
                                                          if captured_cfg else None)),
        "cpu_baseline": cpu,
        "e2e": e2e,
        "fp32_error": err,
        "observer": observed,
        "gpu_launches": launches,
        "clocks": {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"],
                   "samples": clk["samples"]},
    }


def observer_block(args, world, cells, ms, ms_obs, snaps_taken, snaps_dropped):
    """The `observer` object of a Model C line: the same K steps timed with an
    AsyncObserver attached, against `ms` without it."""
    return {"every": args.observe_every, "slots": 3,
            "value": world * cells * args.steps / (ms_obs / 1e3) / 1e9, "unit": "Gcell-updates/s",
            "slowdown": ms_obs / ms - 1.0, "captured": snaps_taken, "dropped": snaps_dropped,
            "snapshot_bytes": 2 * cells * 8,
            "what": "device-timed K steps with the observer attached (gather kernel on the stepping "
                    "stream, copy on the ring's stream, a host thread reducing each snapshot)"}


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="own", choices=["own", "reference"])
    ap.add_argument("--config", default="c3", choices=sorted(CONFIGS))
    ap.add_argument("--dtype", default="f64", choices=["f64", "f32"])
    ap.add_argument("--variant", type=int, default=0)
    ap.add_argument("--noise", type=float, default=None, help="override the noise amplitude b")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cells", type=int, default=None, help="override the grid's cells per dimension (small cases)")
    ap.add_argument("--instances", type=int, default=None, help="override the ensemble's instance count")
    ap.add_argument("--integrator", default="em", choices=["em", "rk4"],
                    help="rk4: RungeKutta4 (deterministic: the noise amplitude is set to 0)")
    ap.add_argument("--observe-every", type=int, default=0,
                    help="also time the run with an AsyncObserver snapshotting phi and u every N steps")
    argv = sys.argv[1:] if argv is None else list(argv)
    args = ap.parse_args(argv)
    args.dtype_given = any(a == "--dtype" or a.startswith("--dtype=") for a in argv)
    args.warmup = max(args.warmup, 3)
    cfg = dict(CONFIGS[args.config])
    if args.noise is not None:
        cfg["noise"] = args.noise
    if args.integrator == "rk4":
        cfg["integrator"] = "rk4"
        cfg["noise"] = 0.0
        cfg["workload"] += "_rk4"
    if args.cells is not None:
        cfg["cells"] = args.cells
        cfg["workload"] += f"_cells{args.cells}"
    if args.instances is not None:
        cfg["instances"] = args.instances
        cfg["workload"] += f"_inst{args.instances}"
    return args, cfg


def main():
    args, cfg = parse_args()
    if args.impl == "reference":
        run_reference(args, cfg)
        return
    if cfg.get("kind") in ("heat", "amr"):
        run_other(args, cfg)
        return
    if cfg.get("kind") == "ensemble":
        run_ensemble(args, cfg)
        return
    run_model_c(args, cfg)


def run_model_c(args, cfg):
    """Uniform-grid Model C (c2, c3, c3o): device-timed K steps, the same K
    steps end to end through the C ABI from pinned host buffers, and the
    optional observer, FP32-error and CPU-baseline legs."""
    import ctypes as C

    import torch

    import legendre_b200 as L

    rank, world, local, pg = dist_setup(args.gpus)
    # a dedicated stream: the library launches on it and the CUDA events
    # below are recorded on it
    stream = torch.cuda.Stream(device=local)
    torch.cuda.set_stream(stream)
    sched = L.CudaScheduler(local, stream.cuda_stream)
    sim, grid, model, grains = make_sim(cfg, args.dtype, sched, seed_offset=rank)
    initialize(sim, grid, model, grains, cfg, args.dtype, sched)
    dt = cfg["dt"]
    cells = cfg["cells"] ** 2

    # the project's autotuner picks the step variant for this shape unless
    # one is forced; warm-up (also captures the step graph)
    tuned = None
    if args.variant == 0 and cfg.get("integrator") != "rk4":  # the tuner times the Euler-Maruyama step
        tuned, _ = sim.autotune(dt, trial_steps=10)
    sim.run(dt, args.warmup, graph=True, variant=args.variant)
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    barrier(pg)
    torch.cuda.synchronize()
    launches0 = sched.kernel_launches
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.run(dt, args.steps, graph=True, variant=args.variant)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(pg)
    clk = clocks.stop()
    launches = sched.kernel_launches - launches0
    ms = max_over_ranks(pg, e0.elapsed_time(e1))

    # end to end through the C ABI: pinned host state in, K steps, state out
    sdtype = torch.float64 if args.dtype == "f64" else torch.float32
    n_el = grid.num_blocks() * grid.block_len(1)
    host_in = [torch.from_numpy(sim.state.download(f).reshape(-1)).pin_memory() for f in ("phi", "u")]
    host_out = [torch.empty(n_el, dtype=sdtype).pin_memory() for _ in range(2)]
    barrier(pg)
    torch.cuda.synchronize()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for f, buf in enumerate(host_in):
        L._native.check(L._native.lib.lg_state_upload_field(sim.state.handle, f, C.c_void_p(buf.data_ptr()), n_el),
                        sched.handle)
    sim.run(dt, args.steps, graph=True, variant=args.variant)
    for f, buf in enumerate(host_out):
        L._native.check(L._native.lib.lg_state_download_field(sim.state.handle, f, C.c_void_p(buf.data_ptr()), n_el),
                        sched.handle)
    e3.record(stream)
    torch.cuda.synchronize()
    barrier(pg)
    ms_e2e = max_over_ranks(pg, e2.elapsed_time(e3))
    esz = 8 if args.dtype == "f64" else 4
    e2e = {"value": world * cells * args.steps / (ms_e2e / 1e3) / 1e9, "unit": "Gcell-updates/s",
           "h2d_bytes_per_step": 2 * n_el * esz / args.steps, "d2h_bytes_per_step": 2 * n_el * esz / args.steps,
           "what": f"lg_state_upload_field x2 from pinned host + {args.steps} steps + lg_state_download_field x2, "
                   "device-timed on the library's stream, bytes amortised per step"}

    # observed: the same K steps with an AsyncObserver taking snapshots of
    # phi and u every N steps into a 3-slot ring; its sink reduces each one on
    # the host (mean phi, solid fraction) while the device keeps stepping
    observed = None
    if args.observe_every > 0:
        class StatsSink:
            def __init__(self):
                self.rows = []

            def consume(self, snap):
                phi = snap.columns["phi"]
                self.rows.append((snap.step, float(phi.mean()), float((phi > 0).mean())))

            def finish(self):
                pass

        sink = StatsSink()
        obs = L.AsyncObserver(every=args.observe_every, nslots=3, sinks=[sink], fields=[("phi", "phi"), ("u", "u")])
        sim.add_observer(obs)
        sim.run(dt, args.observe_every, graph=True, variant=args.variant)  # binds the ring, warms the graphs
        torch.cuda.synchronize()
        barrier(pg)
        e4 = torch.cuda.Event(enable_timing=True)
        e5 = torch.cuda.Event(enable_timing=True)
        e4.record(stream)
        sim.run(dt, args.steps, graph=True, variant=args.variant)
        e5.record(stream)
        torch.cuda.synchronize()
        ms_obs = max_over_ranks(pg, e4.elapsed_time(e5))
        snaps_taken, snaps_dropped = obs.stats()
        obs.close()
        sim.observers.clear()
        observed = observer_block(args, world, cells, ms, ms_obs, snaps_taken, snaps_dropped)

    if rank == 0:
        peak, peak_kind = peaks()
        err = None
        if args.dtype == "f32" and world == 1:
            err = fp32_error(cfg, sched, min(args.steps, cfg["full_steps"]))
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            rate, steps_run, threads, _ = cpu_oracle_rate(cfg, steps_budget_s=15.0, max_steps=1000)
            cpu = {"value": rate, "unit": "Gcell-updates/s", "cores": threads, "kind": "port",
                   "sample": f"{steps_run} steps of the same {cfg['cells']}^2 grid after 1 warm-up step, "
                             "OpenMP over blocks"}
        line = model_c_line(args, cfg, world, ms, clk, launches, tuned, e2e, observed, err, cpu, peak, peak_kind,
                            compute_peaks=sched.compute_peaks())
        print(json.dumps(line), flush=True)
    sched.close()
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
