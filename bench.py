#!/usr/bin/env python
"""Benchmark of the mobydiff RK3 time step on B200.

Default workload (``--config c1``): the wavy-wall channel with immersed
boundary on a 256x128x128 staggered grid (walls y = y0 + A sin(2 pi x /
lambda) and +2, A = 0.05, lambda = Lx/2), Re 3000, dt 1e-3, red-black SOR
(omega 1.7), seeded Poiseuille + noise initial condition projected at
t = 0.  One step = one full RK3 step (3 predictor passes, 3 projections to
tolerance, boundary conditions).  ``value`` is the learned + mixed step:
each projection starts from the extrapolated pressure increment plus the
trained network's correction and runs FP32 sweeps inside FP64 defect
correction to residual 1e-8.  The same run measures the plain FP64 step
(zero start, FP64 sweeps) at residual 1e-8 and at 1e-10, the velocity error
of the learned + mixed state against the plain FP64 one after the same
steps, and the network's training (snapshots recorded by two held-out runs
of the geometry at other seeds and amplitudes).  ``--config c1-plain`` is
the plain FP64 step to 1e-10 alone; ``c0`` and ``c2`` the FFT path.

Prints ONE JSON line on rank 0.  ``value`` is Mcell-steps/s with fields
resident in HBM; ``e2e`` is the same metric through the C ABI with the
state copied host->device and device->host (pinned buffers) every step.
``--impl reference`` times the CPU restatement of the reference (the
oracle: plain FP64 red-black SOR from phi = 0, the reference's method) on
the host cores instead, at the tolerance of the chosen config.

Multi-GPU (torchrun): every rank advances its own replica of the workload
(the step has no exchange between independent channels); value = total
cell-steps of all ranks / max elapsed over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcell-steps/s and Poisson iters to 1e-8: learned+mixed vs plain FP64, 1 B200"
UNIT = "Mcell-steps/s"

C1_GEOM = dict(nx=256, ny=128, nz=128, lx=2 * math.pi, ly=2.25, lz=math.pi, re=3000.0, dt=1e-3, solver="redblack",
               sor=1.7, check_every=50, ibm="wavy", amp=0.05)
CONFIGS = {
    "c1": dict(C1_GEOM, workload="wavy-wall IBM channel 256x128x128 (Re 3000, A 0.05), red-black SOR omega=1.7 to "
                                 "residual 1e-8: learned warm start + FP32 sweeps in FP64 defect correction",
               tol=1e-8, method="learned-mixed"),
    "c1-plain": dict(C1_GEOM, workload="wavy-wall IBM channel 256x128x128, FP64 red-black SOR omega=1.7 to residual "
                                       "1e-10", tol=1e-10, method="plain"),
    "c3": dict(C1_GEOM, workload="learned warm start on the 256x128x128 wavy-wall IBM channel: network trained on "
                                 "snapshots of runs at Re in 1000..5000, A in 0..0.1 (stratified draws); "
                                 "held-out runs at Re U(1000,5000), A U(0,0.1); SOR iterations to residual 1e-8 "
                                 "on held-out runs against zero, previous-step and extrapolated guesses (FP32 sweeps "
                                 "in FP64 defect correction, omega 1.7)",
               tol=1e-8, method="learned-eval", check_every=10, train_runs=8, record_steps=8, heldout_runs=4,
               heldout_steps=10),
    "c4": dict(workload="ensemble of 64 wavy-wall IBM channels, nx,nz in 32..128 and ny in 32..96 (multiples of 16), "
                         "Re U(1000,5000), A U(0,0.1), red-black SOR omega=1.7 to residual 1e-8, FP32 sweeps in FP64 "
                         "defect correction, learned warm start (network trained on stratified member-like runs); "
                         "two persistent launches per RK3 substage with the network between, CUDA graph, autotuned "
                         "launch shape",
               solver="redblack", sor=1.7, tol=1e-8, check_every=25, members=64, method="ensemble", mixed=True,
               learned=True, train_runs=6, record_steps=6),
    "c0": dict(workload="periodic channel 64^3, FP64 FFT+Thomas", nx=64, ny=64, nz=64, lx=2 * math.pi, ly=2.0,
               lz=math.pi, re=2000.0, dt=1e-3, solver="fft", ibm="none", amp=0.0, method="plain"),
    "c2": dict(workload="channel 512x256x256 (Lx 4pi, Lz 2pi, Re 5000): FP32 FFT + Thomas inside FP64 defect "
                         "correction to residual 1e-10, zero-wavenumber mode in FP64",
               nx=512, ny=256, nz=256, lx=4 * math.pi, ly=2.0, lz=2 * math.pi, re=5000.0, dt=1e-3, solver="fft",
               ibm="none", amp=0.0, tol=1e-10, method="fft-mixed"),
    "c2-plain": dict(workload="channel 512x256x256 (Lx 4pi, Lz 2pi, Re 5000), FP64 FFT+Thomas", nx=512, ny=256,
                     nz=256, lx=4 * math.pi, ly=2.0, lz=2 * math.pi, re=5000.0, dt=1e-3, solver="fft", ibm="none",
                     amp=0.0, method="plain"),
}

# Held-out training runs of the learned warm start: (seed, wall amplitude).
TRAIN_RUNS = ((20261204, 0.03), (20261205, 0.07))
# --train-runs 4: wall amplitudes around the timed run's 0.05, none equal to it
TRAIN_RUNS4 = ((20261204, 0.02), (20261205, 0.04), (20261206, 0.06), (20261207, 0.08))
SEED = 20261203


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fp:
            p = json.load(fp)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _traffic_per_cell(kernel: str):
    """DRAM bytes per cell of one launch of `kernel` from the committed ncu summary, or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as fp:
            t = json.load(fp)
        return float(t[kernel]["dram_bytes_per_cell"])
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "samples": len(sm),
                "reasons": sorted(reasons)}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


C3_GATE_PERIOD = 16   # the learned_gated guess re-tries the other choice every 16th projection of a substage
SOR_VARIANT = 0   # --sor-variant: red-black kernel variant (0: the autotuner's choice)
FFT_KERNEL = 0    # --fft-kernel: 0 warp-shuffle transforms where the lengths allow, 1 Stockham
INNER_FORM = 0    # --inner-form: FP32 correction sweeps of the mixed path, 0 potential form, 1 face form
SOR_NAMES = {1: "one launch per colour sweep", 2: "fused red+black pass 32x8", 3: "fused red+black pass 32x16",
             4: "one launch per colour sweep on colour-split copies",
             5: "one launch per colour sweep on colour-split copies, 2 cells per thread"}


# FP32 correction sweeps of the mixed path, by the hundreds digit of the
# solve's variant
SOR32_NAMES = {1: "k_sor_sweep32: one launch per colour, one cell per thread",
               3: "k_rb32_fused: one launch per red+black iteration",
               5: "k_sor_sweep32v: one launch per colour, 2 or 4 cells per thread",
               7: "potential form: the autotuner's pick among k_pot_sweep (2 or 4 cells per thread), k_pot_sweep_w "
                  "(one warp per row), k_pot_sweep_a (planes staged by cp.async) and k_pot_run_w (one warp per row, "
                  "a block of iterations per cooperative launch; the pick on 256x128x128)"}
SOR32_TRAFFIC = {1: "sor_sweep32", 3: "rb32_fused", 5: "sor_sweep32v", 7: "pot_run_w"}
# algorithmic bytes per cell of one FP32 colour sweep launch (a fused
# red+black launch does both colours): the face form reads and writes 4
# floats per cell of one colour (16 B per cell of the grid); the potential
# form reads phi of both colours and r~ of the swept one and writes phi of
# the swept one (8 B per cell of the grid)
SOR32_ALG = {1: 16.0, 3: 32.0, 5: 16.0, 7: 8.0}


def _sor64_traffic_key(variant):
    """traffic.json entry of the FP64 sweep kernel a solve ran."""
    return {4: "sor_sweep_split", 5: "sor_sweep_splitv"}.get(variant, "sor_sweep")


def _setup(cfg, M, device, profile=False, tol=None, precision=None, seed=None):
    g = M.make_grid(cfg["nx"], cfg["ny"], cfg["nz"], cfg["lx"], cfg["ly"], cfg["lz"], cfg["re"], cfg["dt"],
                    (2.0 / cfg["re"], 0.0, 0.0))
    bc = M.channel_bc()
    s = M.Solver(g, bc, device)
    s.enter_field_data()
    y0 = (cfg["ly"] - 2.0) / 2.0
    lam = cfg["lx"] / 2.0
    if cfg["ibm"] == "wavy":
        s.enter_ibm_data(*M.set_ibm_coeff(g, M.ibm_wavy(cfg["amp"], lam, y0)))
    if cfg["solver"] == "redblack" and profile:
        # profiling mode: the full-size state with a fixed 20 sweeps per
        # projection, so that an ncu capture of a few launches ends quickly
        opts = M.make_solver_opts(M.SOLVER_REDBLACK, sor=cfg["sor"], n_iter=20, tol=0.0, sor_variant=SOR_VARIANT)
    elif cfg["solver"] == "redblack":
        opts = M.make_solver_opts(M.SOLVER_REDBLACK, sor=cfg["sor"], tol=cfg["tol"] if tol is None else tol,
                                  check_every=cfg["check_every"], max_iter=400000,
                                  precision=M.PREC_FP64 if precision is None else precision,
                                  sor_variant=SOR_VARIANT, inner_form=INNER_FORM)
    else:
        opts = M.make_solver_opts(M.SOLVER_FFT, tol=cfg.get("tol", 0.0) if precision == M.PREC_MIXED else 0.0,
                                  precision=M.PREC_FP64 if precision is None else precision, fft_kernel=FFT_KERNEL)
    s.init_pressure_solver(opts)
    s.channel_ic(SEED if seed is None else seed, 0.1, 0.01, y0, cfg["amp"], lam)
    return s, g


def _oracle_sample(cfg, threads: int, target_s: float = 12.0):
    """Time the oracle's predictor and red-black sweeps (or FFT projection) on
    the workload.  Returns per-phase seconds."""
    from oracle import oracle as O
    O.build()
    O.set_threads(threads)
    g = O.Grid(cfg["nx"], cfg["ny"], cfg["nz"], cfg["lx"], cfg["ly"], cfg["lz"], cfg["re"], cfg["dt"],
               (2.0 / cfg["re"], 0.0, 0.0))
    bc = O.channel_bc()
    f = O.Fields(g)
    y0 = (cfg["ly"] - 2.0) / 2.0
    lam = cfg["lx"] / 2.0
    if cfg["ibm"] == "wavy":
        O.set_ibm_coeff(g, O.ibm_wavy(cfg["amp"], lam, y0), f)
    O.channel_ic(g, f, SEED, 0.1, 0.01, y0, cfg["amp"], lam)
    f.us[...] = f.un
    f.vs[...] = f.vn
    f.ws[...] = f.wn
    a, b, c = O.rk_coeffs()
    dt = cfg["dt"]
    t0 = time.perf_counter()
    for st in range(3):
        O.momentum(g, bc, f, dt * a[st], dt * b[st], dt * c[st])
    t_mom = (time.perf_counter() - t0) / 3
    out = {"momentum": t_mom}
    if cfg["solver"] == "redblack":
        n = 20
        t0 = time.perf_counter()
        O.pressure_projection_redblack(g, bc, f, dt * c[0], niter=n, sor=cfg["sor"], tol=0.0)
        t_it = (time.perf_counter() - t0) / n
        n2 = max(20, int((target_s - 3 * t_mom) / max(t_it, 1e-6)))
        t0 = time.perf_counter()
        O.pressure_projection_redblack(g, bc, f, dt * c[0], niter=n2, sor=cfg["sor"], tol=0.0)
        out["sor_iter"] = (time.perf_counter() - t0) / n2
        out["sor_iters_sampled"] = n + n2
        t0 = time.perf_counter()
        O.divergence_norms(g, bc, f)
        out["residual"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        O.apply_bc_redblack(g, bc, f)
        out["bc"] = time.perf_counter() - t0
    else:
        t0 = time.perf_counter()
        O.apply_bc(g, f)
        O.pressure_projection_fft(g, f, dt * c[0])
        O.apply_bc(g, f)
        out["projection"] = time.perf_counter() - t0
    return out, g.nx * g.ny * g.nz


def _cpu_step_seconds(cfg, ph, iters_per_step):
    if cfg["solver"] == "redblack":
        checks = iters_per_step / cfg["check_every"] + 3
        return 3 * ph["momentum"] + iters_per_step * ph["sor_iter"] + checks * ph["residual"] + 3 * ph["bc"]
    return 3 * (ph["momentum"] + ph["projection"])


def _cpu_baseline(cfg, iters_per_step):
    threads = os.cpu_count() or 1
    ph, cells = _oracle_sample(cfg, threads)
    per_step = _cpu_step_seconds(cfg, ph, iters_per_step)
    if cfg["solver"] == "redblack":
        sample = (f"3 predictor passes + {ph['sor_iters_sampled']} red-black iterations on the full grid; "
                  f"step time extrapolated to the {iters_per_step:.0f} iterations per step of the plain FP64 "
                  f"method at residual {cfg['tol']:g} (the sweeps are bit-identical, so are the counts)")
    else:
        sample = "one predictor + one FFT projection on the full grid, x3 substages"
    return {"value": cells / per_step / 1e6, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample}


def _oracle_state(cfg, O):
    """The seeded start of the workload on the host, made the way
    mdx_channel_ic makes it on the device: Poiseuille + noise, projected at
    t = 0 with dt_gamma = 1 by the config's own solver (red-black: residual
    checked every `check_every` iterations), then p = 0."""
    g = O.Grid(cfg["nx"], cfg["ny"], cfg["nz"], cfg["lx"], cfg["ly"], cfg["lz"], cfg["re"], cfg["dt"],
               (2.0 / cfg["re"], 0.0, 0.0))
    bc = O.channel_bc()
    f = O.Fields(g)
    y0 = (cfg["ly"] - 2.0) / 2.0
    lam = cfg["lx"] / 2.0
    if cfg["ibm"] == "wavy":
        O.set_ibm_coeff(g, O.ibm_wavy(cfg["amp"], lam, y0), f)
    O.channel_ic(g, f, SEED, 0.1, 0.01, y0, cfg["amp"], lam)
    f.us[...] = f.un
    f.vs[...] = f.vn
    f.ws[...] = f.wn
    ic_iters = 0
    if cfg["solver"] == "redblack":
        _, ic_iters, _ = O.pressure_projection_redblack(g, bc, f, 1.0, sor=cfg["sor"], tol=cfg["tol"],
                                                        max_iter=400000, check_every=cfg["check_every"])
        O.apply_bc_redblack(g, bc, f)
    else:
        O.apply_bc(g, f)
        O.pressure_projection_fft(g, f, 1.0)
        O.apply_bc(g, f)
    f.pn[...] = 0.0
    return g, bc, f, ic_iters


def run_reference(args, cfg):
    """The reference's method on the host cores: the oracle (the CPU
    restatement of the reference's step) runs whole RK3 steps end to end
    from the projected seeded start -- predictor, projection to the
    config's residual with its own checks, boundary conditions -- and the
    line reports the measured Mcell-steps/s.  Red-black: one full step
    (minutes on the host; its iteration count is the GPU plain arm's
    `first_step` count, the sweeps being bit-identical); FFT: up to K full
    steps within about a minute."""
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    from oracle import oracle as O
    O.build()
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    t0 = time.perf_counter()
    g, bc, f, ic_iters = _oracle_state(cfg, O)
    setup_s = time.perf_counter() - t0
    cells = cfg["nx"] * cfg["ny"] * cfg["nz"]
    a, _, _ = O.rk_coeffs()
    extra = {}
    if cfg["solver"] == "redblack":
        t0 = time.perf_counter()
        st, iters = O.run(g, bc, f, cfg["dt"], 1, solver=1, sor=cfg["sor"], tol=cfg["tol"], max_iter=400000,
                          check_every=cfg["check_every"])
        elapsed = time.perf_counter() - t0
        nsteps = 1
        extra = {"iterations_per_step": iters, "status": st, "t0_projection_iterations": ic_iters}
        sample = (f"one full RK3 step of the reference's method (FP64 red-black SOR from phi = 0, omega "
                  f"{cfg['sor']}, residual {cfg['tol']:g} checked every {cfg['check_every']} iterations) on the "
                  f"full {cfg['nx']}x{cfg['ny']}x{cfg['nz']} grid from the projected seeded start: {iters} "
                  f"iterations, timed end to end")
    else:
        nsteps = 0
        t0 = time.perf_counter()
        while nsteps < max(args.steps, 1):
            O.run(g, bc, f, cfg["dt"], 1, solver=0)
            nsteps += 1
            if time.perf_counter() - t0 > 60.0:
                break
        elapsed = time.perf_counter() - t0
        sample = f"{nsteps} full RK3 steps (FP64 FFT + Thomas) on the full grid from the projected seeded start"
    value = cells * nsteps / elapsed / 1e6
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": nsteps, "steps_requested": args.steps, "warmup": 0, "ms_per_step": elapsed * 1e3 / nsteps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": cfg["workload"], "arm": "CPU restatement of the reference (oracle), OpenMP, "
                                                           "plain FP64 method, whole steps timed",
                       "setup_s": setup_s},
            "reference_step": extra,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def max_over_ranks(ms, pg):
    """The slowest rank's time: every rank times its own replica, the job
    took as long as the slowest one (NCCL on the GPU, gloo on the CPU)."""
    import torch
    if pg is None:
        return ms
    dev = "cuda" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(ms)], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def aggregate_value(cells_per_rank, steps, ms_max, world):
    """Whole-job Mcell-steps/s: the cells of every replica times the steps,
    over the slowest rank's time."""
    return world * cells_per_rank * steps / (ms_max / 1e3) / 1e6


def _timed_steps(s, stream, steps, pg=None, timing=0):
    """K steps between events on the solver's stream (barrier + synchronize
    on both sides); returns (ms over ranks, ms of this rank, iterations,
    launches, per-class timing).  timing 1: every 8th launch of each kernel
    class is bracketed by events as well; timing 2: only each run of
    back-to-back red-black sweeps between two residual checks (for the
    roofline; the headline runs without events)."""
    import torch
    s.set_timing(timing)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    launches0 = s.launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    iters = 0
    for _ in range(steps):
        iters += s.step(1)
    ev1.record(stream)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    launches = s.launch_count() - launches0
    ms = ev0.elapsed_time(ev1)
    tim = s.get_timing()
    s.set_timing(False)
    ms_all = ms
    if pg:
        ms_all = max_over_ranks(ms, pg)
    return ms_all, ms, iters, launches, tim


def _e2e_steps(s, stream, host, steps, pg=None):
    """K steps through the C ABI with the state (u, v, w, p) copied from and
    to pinned host buffers every step."""
    import torch
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    iters = 0
    for _ in range(steps):
        s.update_device(*[h.numpy() for h in host])
        iters += s.step(1)
        s.update_host(*[h.numpy() for h in host])
    e1.record(stream)
    torch.cuda.synchronize()
    ems = e0.elapsed_time(e1)
    if pg:
        ems = max_over_ranks(ems, pg)
    return ems, iters


def _roofline(tim, kname, alg_per_cell, cells, ms, traffic_key=None):
    """Dominant kernel against measured HBM.  For the red-black sweeps
    (kname "sor_run") the time is that of whole runs of back-to-back sweep
    launches between residual checks, every run timed with one event pair,
    so the average launch is the sweeps' throughput in the step and the
    runs' share of the replay's time is at most 1."""
    peak, peak_kind = _peaks()
    kms, kn = tim[kname]
    avg_s = (kms / 1e3) / max(kn, 1)
    alg_bytes = alg_per_cell * cells
    achieved = alg_bytes / avg_s / 1e9 if kn else None
    tpc = _traffic_per_cell(traffic_key or kname)
    return {"kernel": traffic_key or kname, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": (achieved / peak) if achieved else None, "peak_kind": peak_kind,
            "traffic": (tpc * cells) if tpc else None, "algorithmic_bytes": alg_bytes,
            "avg_launch_ms": avg_s * 1e3, "launches": kn,
            "timing": ("event pair around each run of back-to-back sweeps" if kname == "sor_run"
                       else "every 8th launch bracketed by events"),
            "share_of_step_time": kms / ms if ms > 0 else None}


def _sor_alg_per_launch(variant, fp32=False):
    """Algorithmic bytes per cell of one sweep launch: 4 arrays read and
    written for the cells of one colour (FP64 32 B, FP32 16 B per cell of
    the grid); a fused red+black launch does both colours."""
    per_colour = 16.0 if fp32 else 32.0
    return 2 * per_colour if variant in (2, 3) else per_colour


def _step_hbm(cells, ms_per_step, iters_per_step, per_iter):
    """The whole red-black step against its algorithmic bytes: 104 B per cell
    per substage for the predictor and projection set-up (13 doubles) and
    `per_iter` B per cell per red+black iteration (64 FP64, 32 FP32 face
    form, 16 FP32 potential form)."""
    peak, peak_kind = _peaks()
    b = cells * (3 * 104.0 + per_iter * iters_per_step)
    gbs = b / (ms_per_step / 1e3) / 1e9
    return {"alg_bytes_per_cell_step": 3 * 104.0 + per_iter * iters_per_step, "formula":
            f"3*104 + {per_iter:g}*iterations per step", "gbs": gbs, "peak_gbs": peak, "frac": gbs / peak,
            "peak_kind": peak_kind}


def _fft_passes(cfg, tim, cells, ms, ms_step):
    """Achieved HBM rate of each pass class of the FP64 FFT projection, from
    its algorithmic bytes per cell: fft_fwd = divergence reads (3 doubles) +
    spectrum write, z transform read+write; thomas = spectrum read+write + the
    two tables; fft_inv = z transform read+write, spectrum read + phi write;
    correct = phi, u*, v*, w*, p read, u, v, w, p write."""
    nx, ny, nz = cfg["nx"], cfg["ny"], cfg["nz"]
    spec = 16.0 * (nx // 2 + 1) / nx                      # bytes of spectrum per cell
    tables = 16.0 * (nx // 2 + 1) * (nz // 2 + 1) * ny / cells
    per_cell = {"fft_fwd": 24.0 + 3 * spec, "thomas": 2 * spec + tables, "fft_inv": 3 * spec + 8.0,
                "correct": 72.0 + (24.0 if cfg["ibm"] != "none" else 0.0)}
    peak, peak_kind = _peaks()
    out = {"peak_gbs": peak, "peak_kind": peak_kind}
    # the whole step against its algorithmic bytes: 29 doubles per cell and
    # substage (predictor 14, x-z FFT 2, Thomas 2, inverse FFT 2, correction 9)
    step_bytes = 3 * 29 * 8.0 * cells
    step_gbs = step_bytes / (ms_step / 1e3) / 1e9
    out["step"] = {"alg_bytes_per_cell_step": 696, "ms_per_step": ms_step, "gbs": step_gbs, "frac": step_gbs / peak}
    nproj = tim["correct"][1]          # one correction launch per projection
    for k, b in per_cell.items():
        kms, kn = tim[k]
        if not kn or not nproj:
            continue
        gbs = b * cells * nproj / (kms / 1e3) / 1e9
        out[k] = {"alg_bytes_per_cell": round(b, 3), "launches": kn, "projections": nproj, "ms": kms, "gbs": gbs,
                  "frac": gbs / peak, "share_of_step_time": kms / ms if ms > 0 else None}
    return out


def _first_step(cfg, M, device, tol):
    """The plain FP64 method's first RK3 step from the projected seeded
    start, residual checked after every `check_every` iterations (the
    oracle's schedule): the same step, start and iteration count as the
    reference arm's timed CPU step."""
    import torch
    s, _ = _setup(cfg, M, device, tol=tol, precision=M.PREC_FP64)
    opts = M.make_solver_opts(M.SOLVER_REDBLACK, sor=cfg["sor"], tol=tol, check_every=cfg["check_every"],
                              max_iter=400000, adaptive_checks=False)
    s.init_pressure_solver(opts)
    s.channel_ic(SEED, 0.1, 0.01, (cfg["ly"] - 2.0) / 2.0, cfg["amp"], cfg["lx"] / 2.0)   # t=0 projection, same checks
    stream = torch.cuda.ExternalStream(s.stream(), device=device)
    ms, _, it, _, _ = _timed_steps(s, stream, 1)
    s.close()
    return {"iterations": it, "ms": ms, "check": f"every {cfg['check_every']} iterations",
            "value": cfg["nx"] * cfg["ny"] * cfg["nz"] / (ms / 1e3) / 1e6, "unit": UNIT}


def _init_dist(device):
    import torch
    ws, rank, local = _dist()
    torch.cuda.set_device(device)
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900),
                                device_id=torch.device("cuda", device))
        return dist
    return None


def run_plain(args, cfg):
    import torch
    import mobydiff_b200 as M

    ws, rank, local = _dist()
    device = local
    pg = _init_dist(device)
    s, g = _setup(cfg, M, device, profile=args.profile)
    cells = cfg["nx"] * cfg["ny"] * cfg["nz"]
    stream = torch.cuda.ExternalStream(s.stream(), device=device)
    if args.profile:
        for _ in range(args.warmup + args.steps):
            s.step(1)
        torch.cuda.synchronize()
        if rank == 0:
            print(json.dumps({"profile_run": cfg["workload"], "launches": s.launch_count()}), flush=True)
        s.close()
        return 0

    for _ in range(args.warmup):
        s.step(1)
    torch.cuda.synchronize()
    # the state at the start of the timed steps, kept on the host so that the
    # end-to-end leg replays exactly the same steps (same iteration counts);
    # at a step boundary u, v, w, p are the whole state (beta_1 = 0,
    # step.f90:22, so oldrhs is not read before it is rewritten)
    host = None
    if not args.no_e2e:
        host = [torch.empty(s.padded, dtype=torch.float64, pin_memory=True) for _ in range(4)]
        s.update_host(*[h.numpy() for h in host])
    clocks = ClockSampler(device)
    clocks.start()
    torch.cuda.nvtx.range_push("value")
    ms_all, ms, iters, launches, _ = _timed_steps(s, stream, args.steps, pg)
    torch.cuda.nvtx.range_pop()
    clk = clocks.stop()
    value = ws * cells * args.steps / (ms_all / 1e3) / 1e6
    e2e_line = None
    if not args.no_e2e:
        ems, e2e_iters = _e2e_steps(s, stream, host, args.steps, pg)
        nbytes = 4 * host[0].numel() * 8
        e2e_line = {"value": ws * cells * args.steps / (ems / 1e3) / 1e6, "unit": UNIT,
                    "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
                    "same_steps_as_value": e2e_iters == iters}
        # the same steps once more with events, for the roofline
        s.update_device(*[h.numpy() for h in host])
    mode = 2 if cfg["solver"] == "redblack" else 1
    _, ms, _, _, tim = _timed_steps(s, stream, args.steps, pg, timing=mode)
    step_hbm = None
    if cfg["solver"] == "redblack":   # 4 doubles per cell per colour sweep
        var = s.last_solve_stats().variant
        roofline = _roofline(tim, "sor_run", _sor_alg_per_launch(var), cells, ms,
                             traffic_key=_sor64_traffic_key(var))
        step_hbm = _step_hbm(cells, ms_all / args.steps, iters / args.steps, 64.0)
    else:
        roofline = _roofline(tim, "momentum", 112.0, cells, ms)   # 14 doubles per cell
    fft_passes = (_fft_passes(cfg, tim, cells, ms, ms_all / args.steps) if cfg["solver"] != "redblack"
                  else None)
    iters_per_substage = iters / (3 * args.steps) if cfg["solver"] == "redblack" else 0
    sor_kernel = None
    if cfg["solver"] == "redblack":
        sor_kernel = SOR_NAMES.get(s.last_solve_stats().variant, "?")
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cpu = _cpu_baseline(cfg, iters / max(args.steps, 1))
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_all / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic: seeded Poiseuille+noise IC (SplitMix64), projected at t=0",
                "config": {"workload": cfg["workload"], "grid": [cfg["nx"], cfg["ny"], cfg["nz"]],
                           "re": cfg["re"], "dt": cfg["dt"], "method": "plain FP64",
                           "parallelism": f"replicas x{ws}",
                           "l2": "inputs larger than L2 (state + IBM coefficients > 126 MB)"},
                "poisson_iters_per_substage": iters_per_substage, "sor_kernel": sor_kernel,
                "roofline": roofline, "step_hbm": step_hbm, "fft_passes": fft_passes, "cpu_baseline": cpu,
                "clocks": clk, "e2e": e2e_line, "gpu_launches": launches}
        print(json.dumps(line), flush=True)
    s.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def _splitmix(state):
    state[0] = (state[0] + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
    z = state[0]
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
    return z ^ (z >> 31)


def ensemble_members(M, n, seed=SEED):
    """Seeded members: nx, nz in {32..128}, ny in {32..96} (multiples of 16),
    Re ~ U(1000, 5000), A ~ U(0, 0.1)."""
    st = [seed]
    u01 = lambda: (_splitmix(st) >> 11) * (1.0 / 9007199254740992.0)
    out = []
    for q in range(n):
        nx = 16 * (2 + _splitmix(st) % 7)
        nz = 16 * (2 + _splitmix(st) % 7)
        ny = 16 * (2 + _splitmix(st) % 5)
        re = 1000.0 + 4000.0 * u01()
        amp = 0.1 * u01()
        out.append(M.make_member(nx, ny, nz, re=re, amp=amp, seed=seed + 1 + q))
    return out


def _train_ensemble_net(M, cfg, device, iters):
    """The learned warm start for the ensemble: snapshots of wavy-channel runs
    on one member-like grid (64x48x64, the members' lengths), Re and A each
    stratified over the members' ranges (1000..5000, 0..0.1), then Adam on
    the device; the network is fully convolutional, so it applies to every
    member's grid."""
    from mobydiff_b200 import learned
    rng = np.random.default_rng(SEED + 4)
    nt = cfg["train_runs"]
    perm = rng.permutation(nt)
    runs = [(SEED + 300 + q, float(0.1 * (q + rng.uniform()) / nt), float(1000.0 + 4000.0 * (perm[q] + rng.uniform()) / nt))
            for q in range(nt)]
    s, g = learned.wavy_solver(64, 48, 64, runs[0][2], runs[0][1], cfg["tol"], check_every=cfg["check_every"],
                               precision=M.PREC_MIXED, device=device)
    net = learned.record_and_train(s, g, runs, warm_steps=3, record_steps=cfg["record_steps"], iters=iters)
    s.close()
    return net


def partition_members(sizes, world):
    """Ensemble members to ranks by cell count: largest first, each to the
    rank with the fewest cells so far (ties: lowest rank).  Deterministic,
    so every rank computes the same split without communicating; the
    members are independent channels, so the ranks exchange nothing."""
    loads = [0] * world
    parts = [[] for _ in range(world)]
    for q in sorted(range(len(sizes)), key=lambda q: (-sizes[q], q)):
        r = min(range(world), key=lambda t: (loads[t], t))
        parts[r].append(q)
        loads[r] += sizes[q]
    return [sorted(p) for p in parts], loads


def run_ensemble(args, cfg):
    import torch
    import mobydiff_b200 as M

    ws, rank, local = _dist()
    device = local
    pg = _init_dist(device)
    all_mems = ensemble_members(M, cfg["members"])
    all_sizes = [m.nx * m.ny * m.nz for m in all_mems]
    cells_total = sum(all_sizes)
    # N ranks: the fixed ensemble split by cell count (strong scaling)
    parts, loads = partition_members(all_sizes, ws)
    mems = [all_mems[q] for q in parts[rank]]
    sizes = [m.nx * m.ny * m.nz for m in mems]
    cells = sum(sizes)
    prec = M.PREC_MIXED if cfg.get("mixed") else M.PREC_FP64
    opts = M.make_solver_opts(M.SOLVER_REDBLACK, sor=cfg["sor"], tol=cfg["tol"], check_every=cfg["check_every"],
                              max_iter=400000, precision=prec)
    W, K = args.warmup, args.steps
    net, train_wall = None, 0.0
    if cfg.get("learned"):
        t0 = time.time()
        net = _train_ensemble_net(M, cfg, device, args.train_iters * 2)
        train_wall = time.time() - t0
    mode = M.GUESS_LEARNED if net else M.GUESS_EXTRAPOLATED
    E = M.Ensemble(mems, opts, device)
    if net:
        E.unet_load(net.params, net.out_scale, channels=net.channels, gate_period=args.c4_gate)
    E.set_guess(mode)
    E.ic()
    cache = os.path.join(os.path.expanduser("~"), ".cache", "mobydiff_b200", "ensemble_tune.json")
    os.makedirs(os.path.dirname(cache), exist_ok=True)
    E.step(W)
    tuned = E.tune(cache)   # times each candidate grid from a saved state, then restores it
    host = {(q, n): E.get(q, n) for q in range(len(mems)) for n in ("un", "vn", "wn", "pn")}
    it0 = [E.member_stats(q)[1] for q in range(len(mems))]
    if pg:
        pg.barrier()
    clocks = ClockSampler(device)
    clocks.start()
    l0 = E.info()["launches"]
    iters = E.step(K)   # device time between events around the K graph replays
    clk = clocks.stop()
    info = E.info()
    launches_timed = info["launches"] - l0
    it_m = [E.member_stats(q)[1] - it0[q] for q in range(len(mems))]
    ms = info["last_step_ms"] * K
    ms_all = ms
    if pg:
        ms_all = max_over_ranks(ms, pg)
    value = cells_total * K / (ms_all / 1e3) / 1e6   # every member of the ensemble, slowest rank's time
    # red-black path algorithmic bytes: 3 x 104 B per cell per step for the
    # predictor and projection set-up, 64 B (FP64) or 32 B (FP32 sweeps) per
    # cell per red+black iteration
    per_it = 32.0 if cfg.get("mixed") else 64.0
    alg = sum(n * (3.0 * 104.0 * K + per_it * it) for n, it in zip(sizes, it_m))
    peak, peak_kind = _peaks()
    achieved = alg / (ms / 1e3) / 1e9
    roofline = {"kernel": "k_ens_substage (whole substage)", "bound": "hbm", "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind, "traffic": None,
                "algorithmic_bytes": alg / K, "avg_launch_ms": ms / (3 * K), "launches": 3 * K}
    learned_info = None
    if net:
        kept, undone, gated = E.unet_stats()
        learned_info = {"corrections_kept": kept, "corrections_undone": undone, "gate_period": args.c4_gate,
                        "left_to_extrapolation_by_gate": gated, "snapshots": net.snapshots,
                        "loss_first": net.loss_first, "loss_last": net.loss_last, "train_ms": net.train_ms,
                        "setup_wall_s": train_wall, "train_runs": [list(r) for r in net.runs],
                        "launches_per_step": launches_timed / max(K, 1)}
    # e2e: the timed steps replayed from the same u, v, w, p, copied from host
    # memory every step through the C ABI (the warm-start history has moved on)
    e2e_line = None
    if not args.no_e2e:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_iters = 0
        for _ in range(K):
            for (q, n), a in host.items():
                E.set(q, n, a)
            e2e_iters += E.step(1)
            for (q, n) in host:
                E.get(q, n)
        e2e_s = time.perf_counter() - t0
        if pg:
            e2e_s = max_over_ranks(e2e_s * 1e3, pg) / 1e3
        nbytes = sum(a.nbytes for a in host.values())
        e2e_line = {"value": cells_total * K / e2e_s / 1e6, "unit": UNIT, "h2d_bytes_per_step": nbytes,
                    "d2h_bytes_per_step": nbytes, "timer": "host wall clock around the C-ABI calls",
                    "same_steps_as_value": False, "iterations": e2e_iters}
    # the same members and steps from the extrapolated increment alone
    no_net = None
    if net:
        E.close()
        X = M.Ensemble(mems, opts, device)
        X.set_guess(M.GUESS_EXTRAPOLATED)
        X.ic()
        X.step(W)
        X.tune(cache)
        if pg:
            pg.barrier()
        x_iters = X.step(K)
        x_ms = X.info()["last_step_ms"] * K
        x_all = max_over_ranks(x_ms, pg) if pg else x_ms
        no_net = {"value": cells_total * K / (x_all / 1e3) / 1e6, "unit": UNIT, "ms_per_step": x_all / K,
                  "poisson_iters_per_member_substage": x_iters / (3 * K * len(mems)),
                  "note": "same members, steps and launch-shape tuning, extrapolated increment only"}
        E = X
    # the same members one after another through single contexts
    seq = None
    if not args.quick and ws == 1:
        seq_ms, seq_iters = 0.0, 0
        for m in mems:
            g = M.make_grid(m.nx, m.ny, m.nz, m.lx, m.ly, m.lz, m.re, m.dt, (2.0 / m.re, 0.0, 0.0))
            s = M.Solver(g, M.channel_bc(), device)
            s.enter_field_data()
            y0, lam = (m.ly - 2.0) / 2.0, m.lx / 2.0
            if m.amp > 0.0:
                s.enter_ibm_data(*M.set_ibm_coeff(g, M.ibm_wavy(m.amp, lam, y0)))
            s.init_pressure_solver(opts)
            s.set_pressure_guess(M.GUESS_EXTRAPOLATED, record=True)
            s.channel_ic(m.seed, 0.1, 0.01, y0, m.amp, lam)
            s.step(W)
            stream = torch.cuda.ExternalStream(s.stream(), device=device)
            ms1, _, it1, _, _ = _timed_steps(s, stream, K)
            seq_ms += ms1
            seq_iters += it1
            s.close()
        seq = {"value": cells * K / (seq_ms / 1e3) / 1e6, "unit": UNIT, "ms_per_step": seq_ms / K,
               "iterations": seq_iters, "ensemble_iterations": iters, "precision": "same as the ensemble"}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": K, "warmup": W,
                "ms_per_step": ms_all / K, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
                "dtype": "f64+f32 (FP32 sweeps in FP64 defect correction)" if cfg.get("mixed") else "f64",
                "data": "synthetic: 64 seeded members (SplitMix64 sizes, Re, A, IC seeds)",
                "config": {"workload": cfg["workload"], "members": len(all_mems), "cells": cells_total,
                           "tol": cfg["tol"],
                           "parallelism": f"members split over {ws} ranks by cell count" if ws > 1 else "1 GPU",
                           "rank_cells": loads, "rank0_members": len(mems),
                           "l2": "inputs larger than L2 (64 members' state > 126 MB)"},
                "poisson_iters_per_member_substage": iters / (3 * K * len(mems)),
                "ensemble": {"threads": info["threads"], "grid": info["grid"], "cuda_graph": info["graph"],
                             "low_regs": info["low_regs"],
                             "autotuned": {"threads": tuned[0], "blocks_per_sm": tuned[1], "low_regs": tuned[2],
                                           "step_ms": tuned[3] if tuned[3] >= 0 else "from cache"},
                             "launches_per_step": 3},
                "sequential_single_contexts": seq,
                "learned": learned_info, "extrapolated_no_network": no_net,
                "roofline": roofline, "cpu_baseline": None, "clocks": clk, "e2e": e2e_line,
                "gpu_launches": launches_timed}
        print(json.dumps(line), flush=True)
    E.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def run_fft_mixed(args, cfg):
    """The FFT path in mixed precision beside the plain FP64 FFT path, on the
    same seeded start and the same steps."""
    import torch
    import mobydiff_b200 as M

    ws, rank, local = _dist()
    device = local
    pg = _init_dist(device)
    cells = cfg["nx"] * cfg["ny"] * cfg["nz"]
    W, K = args.warmup, args.steps
    # plain FP64 FFT arm (CUDA-graph steps)
    sp, _ = _setup(cfg, M, device, precision=M.PREC_FP64)
    stream_p = torch.cuda.ExternalStream(sp.stream(), device=device)
    for _ in range(W):
        sp.step(1)
    p_ms_all, _, _, _, _ = _timed_steps(sp, stream_p, K, pg)
    plain_value = ws * cells * K / (p_ms_all / 1e3) / 1e6
    plain_state = {n: sp.get(n) for n in ("un", "vn", "wn", "pn")}
    sp.close()
    # mixed arm
    s, _ = _setup(cfg, M, device, precision=M.PREC_MIXED)
    stream = torch.cuda.ExternalStream(s.stream(), device=device)
    for _ in range(W):
        s.step(1)
    host = [torch.empty(s.padded, dtype=torch.float64, pin_memory=True) for _ in range(4)]
    s.update_host(*[h.numpy() for h in host])
    clocks = ClockSampler(device)
    clocks.start()
    torch.cuda.nvtx.range_push("value")
    ms_all, ms, passes, launches, _ = _timed_steps(s, stream, K, pg)
    torch.cuda.nvtx.range_pop()
    clk = clocks.stop()
    value = ws * cells * K / (ms_all / 1e3) / 1e6
    interior = (slice(1, -1), slice(1, -1), slice(1, -1))
    err = {n: float(np.linalg.norm((s.get(n) - plain_state[n])[interior]) / np.linalg.norm(plain_state[n][interior]))
           for n in ("un", "vn", "wn", "pn")}
    l2, linf = s.divergence_norms()
    e2e_line = None
    if not args.no_e2e:
        ems, e2e_passes = _e2e_steps(s, stream, host, K, pg)
        nbytes = 4 * host[0].numel() * 8
        e2e_line = {"value": ws * cells * K / (ems / 1e3) / 1e6, "unit": UNIT, "h2d_bytes_per_step": nbytes,
                    "d2h_bytes_per_step": nbytes, "same_steps_as_value": e2e_passes == passes}
    s.update_device(*[h.numpy() for h in host])
    _, r_ms, _, _, tim = _timed_steps(s, stream, K, pg, timing=True)
    roofline = _roofline(tim, "momentum", 112.0, cells, r_ms)   # 14 doubles per cell
    shares = {k: v[0] / r_ms for k, v in tim.items() if v[1]}
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cpu = _cpu_baseline(cfg, 0.0)
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": K, "warmup": W,
                "ms_per_step": ms_all / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64+f32 (FP32 FFT and Thomas in FP64 defect correction)",
                "data": "synthetic: seeded Poiseuille+noise IC (SplitMix64), projected at t=0",
                "config": {"workload": cfg["workload"], "grid": [cfg["nx"], cfg["ny"], cfg["nz"]], "re": cfg["re"],
                           "dt": cfg["dt"], "tol": cfg["tol"], "parallelism": f"replicas x{ws}",
                           "l2": "inputs larger than L2 (state > 126 MB)"},
                "defect_correction_passes_per_substage": passes / (3 * K),
                "plain_fp64": {"value": plain_value, "unit": UNIT, "ms_per_step": p_ms_all / K,
                               "note": "direct FP64 solve, CUDA-graph steps"},
                "speedup_vs_plain_fp64": value / plain_value,
                "error_vs_plain_fp64": {"rel_l2_interior": err, "div_l2": l2, "div_linf": linf},
                "kernel_class_shares": shares,
                "roofline": roofline, "cpu_baseline": cpu, "clocks": clk, "e2e": e2e_line, "gpu_launches": launches}
        print(json.dumps(line), flush=True)
    s.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def run_profile_mixed(args, cfg):
    """Only the set-up: the t=0 projection of the full-size workload with
    FP32 sweeps in FP64 defect correction (for an ncu capture of a few
    FP32 sweep launches)."""
    import torch
    import mobydiff_b200 as M
    _, rank, local = _dist()
    torch.cuda.set_device(local)
    s, _ = _setup(cfg, M, local, tol=1e-8, precision=M.PREC_MIXED)
    torch.cuda.synchronize()
    if rank == 0:
        print(json.dumps({"profile_run": cfg["workload"] + "; t=0 projection, FP32 sweeps",
                          "launches": s.launch_count()}), flush=True)
    s.close()
    return 0


def run_profile_ensemble(args, cfg):
    """The first N members of the C4 ensemble (extrapolated start, FP32 sweeps
    in FP64 defect correction, residual 1e-8), 3 warm-up steps and 2 more, no
    autotuning (for an ncu capture of one substage launch); prints each
    member's iterations over the last 2 steps."""
    import torch
    import mobydiff_b200 as M
    _, rank, local = _dist()
    torch.cuda.set_device(local)
    n = args.profile_ensemble
    mems = ensemble_members(M, n)
    opts = M.make_solver_opts(M.SOLVER_REDBLACK, sor=cfg["sor"], tol=cfg["tol"], check_every=cfg["check_every"],
                              max_iter=400000, precision=M.PREC_MIXED)
    E = M.Ensemble(mems, opts, local)
    E.set_guess(M.GUESS_EXTRAPOLATED)
    E.ic()
    E.step(3)
    it0 = [E.member_stats(q)[1] for q in range(n)]
    E.step(2)
    its = [E.member_stats(q)[1] - it0[q] for q in range(n)]
    info = E.info()
    E.close()
    if rank == 0:
        print(json.dumps({"profile_run": f"first {n} members of the C4 ensemble, 3 + 2 steps",
                          "cells": sum(m.nx * m.ny * m.nz for m in mems), "iters_per_member_2_steps": its,
                          "threads": info.get("threads"), "grid": info.get("grid")}), flush=True)
    return 0


def run_profile_unet(args, cfg):
    """One forward + backward pass of the learned warm start's network on
    random inputs of the workload's grid (for an ncu capture of a few
    convolution launches; no solver steps)."""
    import torch
    import mobydiff_b200 as M
    _, rank, local = _dist()
    torch.cuda.set_device(local)
    g = M.make_grid(cfg["nx"], cfg["ny"], cfg["nz"], cfg["lx"], cfg["ly"], cfg["lz"], cfg["re"], cfg["dt"],
                    (2.0 / cfg["re"], 0.0, 0.0))
    s = M.Solver(g, M.channel_bc(), local)
    s.enter_field_data()
    s.unet_create(channels=32, capacity=0, slope=0.1)
    n = cfg["nx"] * cfg["ny"] * cfg["nz"]
    rng = np.random.default_rng(SEED)
    loss, _, _ = s.unet_loss_grad(rng.standard_normal((M.UNET_INPUTS, n)).astype(np.float32),
                                  rng.standard_normal(n).astype(np.float32))
    st = s.unet_stats()
    if rank == 0:
        print(json.dumps({"profile_run": cfg["workload"] + "; one network forward + backward", "loss": loss,
                          "tcgen05_convolutions": int(st.tc_convs), "launches": s.launch_count()}), flush=True)
    s.close()
    return 0


def run_learned_eval(args, cfg):
    """Config 3: the network trained on snapshots of runs over a range of Re
    and wall amplitudes, judged by red-black iterations to the tolerance on
    held-out runs against the guesses without it."""
    import torch
    import mobydiff_b200 as M
    from mobydiff_b200 import learned

    _, rank, local = _dist()
    torch.cuda.set_device(local)
    rng = np.random.default_rng(SEED + 3)
    # training runs: Re and A each stratified over their range (one draw per
    # stratum, Re strata in a seeded random order), so that a few runs cover
    # both ranges; held-out runs: independent uniform draws
    nt = cfg["train_runs"]
    perm = rng.permutation(nt)
    train = [(SEED + 100 + q, float(0.1 * (q + rng.uniform()) / nt),
              float(1000.0 + 4000.0 * (perm[q] + rng.uniform()) / nt)) for q in range(nt)]   # (seed, A, Re)
    held = [(SEED + 200 + q, float(rng.uniform(0.0, 0.1)), float(rng.uniform(1000.0, 5000.0)))
            for q in range(args.c3_heldout or cfg["heldout_runs"])]
    steps = args.c3_steps or cfg["heldout_steps"]
    cells = cfg["nx"] * cfg["ny"] * cfg["nz"]
    y0 = (cfg["ly"] - 2.0) / 2.0
    lam = cfg["lx"] / 2.0

    def solver(re, amp):
        g = M.make_grid(cfg["nx"], cfg["ny"], cfg["nz"], cfg["lx"], cfg["ly"], cfg["lz"], re, cfg["dt"],
                        (2.0 / re, 0.0, 0.0))
        s = M.Solver(g, M.channel_bc(), local)
        s.enter_field_data()
        if amp > 0.0:
            s.enter_ibm_geometry(M.ibm_wavy(amp, lam, y0))
        s.init_pressure_solver(M.make_solver_opts(M.SOLVER_REDBLACK, sor=cfg["sor"], tol=cfg["tol"],
                                                  check_every=cfg["check_every"], max_iter=400000,
                                                  precision=M.PREC_MIXED, inner_form=INNER_FORM))
        return s, g

    t0 = time.time()
    st_, gt = solver(train[0][2], train[0][1])
    net = learned.record_and_train(st_, gt, train, warm_steps=3, record_steps=cfg["record_steps"],
                                   iters=args.train_iters * 2)
    st_.close()
    train_wall = time.time() - t0

    # "learned": the correction as predicted, kept when it lowers ||div u||;
    # "learned_gated": the same, applied per RK substage only while it takes
    # fewer iterations than the extrapolated guess alone (gate period 16);
    # "learned_energy": scaled by its energy-optimal step, kept when that is > 0
    all_modes = {"zero": M.GUESS_ZERO, "previous": M.GUESS_PREVIOUS, "extrapolated": M.GUESS_EXTRAPOLATED,
                 "learned": M.GUESS_LEARNED, "learned_gated": M.GUESS_LEARNED, "learned_energy": M.GUESS_LEARNED}
    modes = [(m, all_modes[m]) for m in args.c3_guesses.split(",")]
    per_run, totals = [], {m: [0, 0.0] for m, _ in modes}
    for seed, amp, re in held:
        row = {"seed": seed, "re": re, "amp": amp}
        final = {}
        for name, mode in modes:
            s, g = solver(re, amp)
            if mode == M.GUESS_LEARNED:
                learned.load_into(s, net, step_rule=1 if name == "learned_energy" else 0,
                                  gate_period=C3_GATE_PERIOD if name == "learned_gated" else 0)
            s.set_pressure_guess(mode, record=True)
            s.channel_ic(seed, 0.1, 0.01, y0, amp, lam)
            s.step(3)
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            it = s.step(steps)
            dt = time.perf_counter() - t1
            row[name] = {"iters_per_substage": it / (3 * steps), "mcell_steps_s": cells * steps / dt / 1e6}
            totals[name][0] += it
            totals[name][1] += dt
            if name == "learned_gated":
                row[name]["gated_off"] = s.unet_stats().gated
            final[name] = [s.get(n) for n in ("un", "vn", "wn")]
            s.close()
        ref_name = "zero" if "zero" in final else "extrapolated"
        for name in final:
            if name.startswith("learned"):
                num = sum(float(np.sum((a - b) ** 2)) for a, b in zip(final[name], final[ref_name]))
                den = sum(float(np.sum(b ** 2)) for b in final[ref_name])
                row[f"velocity_rel_l2_{name}_vs_{ref_name}"] = math.sqrt(num / den)
        per_run.append(row)
    nsub = 3 * steps * len(held)
    summary = {m: {"iters_per_substage": totals[m][0] / nsub,
                   "mcell_steps_s": cells * steps * len(held) / totals[m][1] / 1e6} for m, _ in modes}
    head = "learned" if "learned" in summary else "learned_gated"
    ratios = {f"reduction_vs_{b}": summary[b]["iters_per_substage"] / summary[head]["iters_per_substage"]
              for b in ("zero", "previous", "extrapolated") if b in summary}
    for m in ("learned_gated", "learned_energy"):
        if m in summary and m != head and "extrapolated" in summary:
            ratios[f"{m}_reduction_vs_extrapolated"] = (summary["extrapolated"]["iters_per_substage"] /
                                                        summary[m]["iters_per_substage"])
    if rank == 0:
        print(json.dumps({
            "metric": "red-black iterations per substage to residual 1e-8 on held-out runs, learned warm start vs "
                      "zero / previous / extrapolated guesses, 1 B200",
            "value": summary[head]["iters_per_substage"], "unit": "iterations per substage", "value_guess": head,
            "higher_is_better": False, "n_gpus": 1, "steps": steps, "warmup": 3, "dtype": "f64+f32",
            "data": "synthetic: seeded Poiseuille+noise ICs; training and held-out runs at seeded Re and A",
            "config": {"workload": cfg["workload"], "grid": [cfg["nx"], cfg["ny"], cfg["nz"]], "tol": cfg["tol"],
                       "train_runs": [{"seed": a, "amp": b, "re": c} for a, b, c in train],
                       "record_steps_per_run": cfg["record_steps"], "heldout_steps": steps * len(held)},
            "by_guess": summary, **ratios,
            "gate_period": C3_GATE_PERIOD,
            "heldout_runs": per_run,
            "learned": {"snapshots": net.snapshots, "loss_first": net.loss_first, "loss_last": net.loss_last,
                        "train_ms": net.train_ms, "record_s": net.record_seconds, "setup_wall_s": train_wall},
        }), flush=True)
    return 0


def run_learned_mixed(args, cfg):
    import torch
    import mobydiff_b200 as M
    from mobydiff_b200 import learned

    ws, rank, local = _dist()
    device = local
    pg = _init_dist(device)
    cells = cfg["nx"] * cfg["ny"] * cfg["nz"]
    tol = cfg["tol"]
    W, K = args.warmup, args.steps

    # ---- plain FP64 arm: zero start, FP64 sweeps, same tolerance ------------
    first_step = _first_step(cfg, M, device, tol)
    sp, g = _setup(cfg, M, device, tol=tol, precision=M.PREC_FP64)
    stream_p = torch.cuda.ExternalStream(sp.stream(), device=device)
    for _ in range(W):
        sp.step(1)
    p_ms_all, p_ms, p_iters, _, _ = _timed_steps(sp, stream_p, K, pg)
    plain_value = ws * cells * K / (p_ms_all / 1e3) / 1e6
    plain_state = {n: sp.get(n) for n in ("un", "vn", "wn", "pn")}
    # one more step with the sweep runs timed, for the FP64 sweep's roofline
    _, r_ms, _, _, p_tim = _timed_steps(sp, stream_p, 1, pg, timing=2)
    var64 = sp.last_solve_stats().variant
    roof64 = _roofline(p_tim, "sor_run", _sor_alg_per_launch(var64), cells, r_ms,
                       traffic_key=_sor64_traffic_key(var64))
    roof64["sor_kernel"] = SOR_NAMES.get(var64, "?")
    plain_step_hbm = _step_hbm(cells, p_ms_all / K, p_iters / K, 64.0)
    plain_c1 = None
    if not args.quick:   # the plain FP64 step at the C1 tolerance 1e-10
        sp.init_pressure_solver(M.make_solver_opts(M.SOLVER_REDBLACK, sor=cfg["sor"], tol=1e-10,
                                                   check_every=cfg["check_every"], max_iter=400000))
        y0 = (cfg["ly"] - 2.0) / 2.0
        sp.channel_ic(SEED, 0.1, 0.01, y0, cfg["amp"], cfg["lx"] / 2.0)
        for _ in range(W):
            sp.step(1)
        c_ms_all, _, c_iters, _, _ = _timed_steps(sp, stream_p, K, pg)
        plain_c1 = {"value": ws * cells * K / (c_ms_all / 1e3) / 1e6, "unit": UNIT, "tol": 1e-10,
                    "poisson_iters_per_substage": c_iters / (3 * K), "ms_per_step": c_ms_all / K}
    sp.close()

    # ---- training: snapshots of two held-out runs, Adam on the device --------
    t0 = time.time()
    st_, gt = learned.wavy_solver(cfg["nx"], cfg["ny"], cfg["nz"], cfg["re"], cfg["amp"], tol,
                                  check_every=cfg["check_every"], precision=M.PREC_MIXED, device=device,
                                  ly=cfg["ly"], lx=cfg["lx"], lz=cfg["lz"], dt=cfg["dt"])
    runs = TRAIN_RUNS4 if args.train_runs == 4 else TRAIN_RUNS
    net = learned.record_and_train(st_, gt, runs, warm_steps=3, record_steps=16 if len(runs) == 2 else 12,
                                   iters=args.train_iters)
    st_.close()
    train_wall = time.time() - t0

    # ---- learned + mixed arm ----------------------------------------------------
    s, g = _setup(cfg, M, device, tol=tol, precision=M.PREC_MIXED)
    learned.load_into(s, net)
    s.set_pressure_guess(M.GUESS_LEARNED, record=True)
    stream = torch.cuda.ExternalStream(s.stream(), device=device)
    for _ in range(W):
        s.step(1)
    # the state at the start of the timed steps: u, v, w, p on the host, the
    # warm-start history in a device checkpoint, so that the end-to-end leg
    # and the arm without the network replay exactly the same steps
    host = [torch.empty(s.padded, dtype=torch.float64, pin_memory=True) for _ in range(4)]
    s.update_host(*[h.numpy() for h in host])
    s.warm_checkpoint()
    u0 = s.unet_stats()
    clocks = ClockSampler(device)
    clocks.start()
    torch.cuda.nvtx.range_push("value")   # the region an ncu launch list filters on (--nvtx-include "value/")
    ms_all, ms, iters, launches, _ = _timed_steps(s, stream, K, pg)
    torch.cuda.nvtx.range_pop()
    clk = clocks.stop()
    u1 = s.unet_stats()
    value = ws * cells * K / (ms_all / 1e3) / 1e6
    err = {n: float(np.linalg.norm(s.get(n) - plain_state[n]) / np.linalg.norm(plain_state[n]))
           for n in ("un", "vn", "wn", "pn")}
    vnum = sum(float(np.sum((s.get(n) - plain_state[n]) ** 2)) for n in ("un", "vn", "wn"))
    vden = sum(float(np.sum(plain_state[n] ** 2)) for n in ("un", "vn", "wn"))
    err["velocity"] = math.sqrt(vnum / vden)
    # pressure is defined up to a constant (no projection fixes its mean):
    # the error of p with each field's interior mean removed, and that mean's
    # difference
    inner = (slice(1, -1),) * 3
    pa, pb = plain_state["pn"][inner], s.get("pn")[inner]
    err["pn_zero_mean"] = float(np.linalg.norm((pb - pb.mean()) - (pa - pa.mean())) /
                                np.linalg.norm(pa - pa.mean()))
    err["pn_mean_difference"] = float(pb.mean() - pa.mean())
    ls = s.last_solve_stats()
    l2, linf = s.divergence_norms()

    # ---- end to end: the same K steps through the C ABI with host buffers ----
    e2e_line = None
    if not args.no_e2e:
        s.warm_checkpoint(restore=True)
        ems, e2e_iters = _e2e_steps(s, stream, host, K, pg)
        nbytes = 4 * host[0].numel() * 8
        e2e_line = {"value": ws * cells * K / (ems / 1e3) / 1e6, "unit": UNIT, "h2d_bytes_per_step": nbytes,
                    "d2h_bytes_per_step": nbytes, "same_steps_as_value": e2e_iters == iters}

    # ---- the same steps with the sweep runs timed, for the roofline ------------
    s.warm_checkpoint(restore=True)
    s.update_device(*[h.numpy() for h in host])
    _, r_ms, _, _, tim = _timed_steps(s, stream, K, pg, timing=2)
    # 4 floats per cell per colour sweep; the FP32 sweep kernel the autotuner
    # kept is the hundreds digit of the solve's variant
    kind = s.last_solve_stats().variant // 100
    roofline = _roofline(tim, "sor_run", SOR32_ALG.get(kind, 16.0), cells, r_ms,
                         traffic_key=SOR32_TRAFFIC.get(kind, "sor_sweep32"))
    roofline["sor_kernel"] = SOR32_NAMES.get(kind, "?")
    if kind == 7:
        roofline["note"] = ("phi and r~ (37 MB) stay resident in the 126 MB L2 across sweeps, so the sweeps "
                            "run from L2 and can pass the HBM copy rate")
    step_hbm = _step_hbm(cells, ms_all / K, iters / K, 16.0 if kind == 7 else 32.0)

    # ---- the same steps without the network: extrapolated increment only ----
    s.warm_checkpoint(restore=True)
    s.update_device(*[h.numpy() for h in host])
    s.set_pressure_guess(M.GUESS_EXTRAPOLATED, record=True)
    x_ms_all, _, x_iters, _, _ = _timed_steps(s, stream, K, pg)
    no_net = {"value": ws * cells * K / (x_ms_all / 1e3) / 1e6, "unit": UNIT, "ms_per_step": x_ms_all / K,
              "poisson_iters_per_substage": x_iters / (3 * K)}
    s.close()

    # ---- the relaxation factor's share, measured apart: learned + mixed with
    # the FP32 correction sweeps at omega 1.95 (the FP64 test unchanged), and
    # the plain FP64 method with omega 1.95 as its input, same start and steps
    tuned = None
    if not args.quick:
        om = 1.95
        st2, _ = _setup(cfg, M, device, tol=tol, precision=M.PREC_MIXED)
        st2.init_pressure_solver(M.make_solver_opts(M.SOLVER_REDBLACK, sor=cfg["sor"], tol=tol,
                                                    check_every=cfg["check_every"], max_iter=400000,
                                                    precision=M.PREC_MIXED, inner_sor=om,
                                                    inner_form=INNER_FORM))
        st2.channel_ic(SEED, 0.1, 0.01, (cfg["ly"] - 2.0) / 2.0, cfg["amp"], cfg["lx"] / 2.0)
        learned.load_into(st2, net)
        st2.set_pressure_guess(M.GUESS_LEARNED, record=True)
        for _ in range(W):
            st2.step(1)
        t_ms_all, _, t_iters, _, _ = _timed_steps(st2, torch.cuda.ExternalStream(st2.stream(), device=device), K, pg)
        st2.close()
        cfg_om = dict(cfg, sor=om)
        sp2, _ = _setup(cfg_om, M, device, tol=tol, precision=M.PREC_FP64)
        for _ in range(W):
            sp2.step(1)
        q_ms_all, _, q_iters, _, _ = _timed_steps(sp2, torch.cuda.ExternalStream(sp2.stream(), device=device), K, pg)
        sp2.close()
        tuned = {"omega": om,
                 "learned_mixed_inner_omega": {"value": ws * cells * K / (t_ms_all / 1e3) / 1e6, "unit": UNIT,
                                               "poisson_iters_per_substage": t_iters / (3 * K)},
                 "plain_fp64_omega": {"value": ws * cells * K / (q_ms_all / 1e3) / 1e6, "unit": UNIT,
                                      "poisson_iters_per_substage": q_iters / (3 * K)}}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cpu = _cpu_baseline(cfg, p_iters / max(K, 1))
    if rank == 0:
        corr = u1.corrections - u0.corrections
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": K, "warmup": W,
                "ms_per_step": ms_all / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64+f32 (FP32 sweeps in FP64 defect correction; BF16/FP32 network)",
                "data": "synthetic: seeded Poiseuille+noise IC (SplitMix64), projected at t=0; network trained on "
                        "snapshots of two runs at other seeds and wall amplitudes",
                "config": {"workload": cfg["workload"], "grid": [cfg["nx"], cfg["ny"], cfg["nz"]], "re": cfg["re"],
                           "dt": cfg["dt"], "tol": tol, "method": "learned warm start + mixed precision",
                           "parallelism": f"replicas x{ws}",
                           "l2": "inputs larger than L2 (state + IBM coefficients > 126 MB)"},
                "poisson_iters_per_substage": iters / (3 * K),
                "plain_fp64": {"value": plain_value, "unit": UNIT, "tol": tol, "ms_per_step": p_ms_all / K,
                               "poisson_iters_per_substage": p_iters / (3 * K), "roofline": roof64,
                               "step_hbm": plain_step_hbm, "first_step": first_step},
                "plain_fp64_c1_tol": plain_c1,
                "extrapolated_mixed_no_network": no_net,
                "relaxation_tuned": tuned,
                "speedup_vs_plain_fp64": value / plain_value,
                "error_vs_plain_fp64": {"rel_l2": err, "residual": ls.residual, "div_l2": l2, "div_linf": linf},
                "learned": {"corrections": corr, "rejected": u1.rejected - u0.rejected,
                            "divergence_gain_last": u1.last_gain, "inference_ms": u1.infer_ms,
                            "snapshots": net.snapshots, "loss_first": net.loss_first, "loss_last": net.loss_last,
                            "record_s": net.record_seconds, "train_ms": net.train_ms, "setup_wall_s": train_wall,
                            "train_runs": [list(r) for r in runs]},
                "roofline": roofline, "step_hbm": step_hbm, "cpu_baseline": cpu, "clocks": clk, "e2e": e2e_line,
                "gpu_launches": launches}
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    # 5 warm-up steps put the timed steps past the start-up transient of the
    # warm starts (the first steps after the t=0 projection take 2-3x the
    # iterations); 20 timed steps of the headline take about 3 s
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c1", choices=sorted(CONFIGS))
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg")
    ap.add_argument("--profile", action="store_true",
                    help="profiling run for ncu: full-size state, fixed 20 red-black iterations per projection")
    ap.add_argument("--profile-unet", action="store_true",
                    help="one network forward + backward on the workload's grid (for an ncu capture)")
    ap.add_argument("--profile-ensemble", type=int, default=0, metavar="N",
                    help="profiling run for ncu: the first N members of the C4 ensemble, 3 + 2 steps")
    ap.add_argument("--profile-mixed", action="store_true",
                    help="profiling run for ncu: the full-size t=0 projection with FP32 sweeps to residual 1e-8")
    ap.add_argument("--quick", action="store_true", help="skip the plain FP64 leg at residual 1e-10")
    ap.add_argument("--sor-variant", type=int, default=0, choices=list(range(16)),
                    help="red-black kernel variant (0: autotuned; all give the same bits); FP64 sweeps and the "
                         "face form 1-5, the potential form's sweep shapes 1-15")
    ap.add_argument("--inner-form", type=int, default=0, choices=[0, 1, 2],
                    help="mixed red-black: FP32 correction sweeps in the potential form (0; the ensemble keeps the "
                         "face form), the face form (1), or the potential form in the ensemble too (2)")
    ap.add_argument("--fft-kernel", type=int, default=0, choices=[0, 1],
                    help="FFT path transforms: 0 warp-shuffle where nx/2 and nz allow, 1 shared-memory Stockham")
    ap.add_argument("--c3-steps", type=int, default=0,
                    help="config c3: measured steps per held-out run (0: the config's 10)")
    ap.add_argument("--check-every", type=int, default=0,
                    help="red-black: iterations between residual checks (0: the config's)")
    ap.add_argument("--c4-gate", type=int, default=0,
                    help="config c4: gate period of the learned correction per member (0, the default: no gate)")
    ap.add_argument("--c3-heldout", type=int, default=0,
                    help="config c3: held-out runs (0: the config's 4; the first 4 draws are the same either way)")
    ap.add_argument("--c3-guesses", default="zero,previous,extrapolated,learned,learned_gated",
                    help="config c3: the guesses compared (comma list of zero, previous, extrapolated, learned, "
                         "learned_gated, learned_energy)")
    ap.add_argument("--train-iters", type=int, default=1200, help="Adam steps of the learned warm start")
    ap.add_argument("--train-runs", type=int, default=2, choices=[2, 4],
                    help="headline: training runs of the learned warm start (2: A 0.03, 0.07; 4: A 0.02..0.08)")
    args = ap.parse_args()
    global SOR_VARIANT, FFT_KERNEL, INNER_FORM
    SOR_VARIANT = args.sor_variant
    INNER_FORM = args.inner_form
    FFT_KERNEL = args.fft_kernel
    cfg = CONFIGS[args.config]
    if args.check_every > 0:
        cfg = dict(cfg, check_every=args.check_every)
    if args.impl == "reference":
        return run_reference(args, cfg)
    if args.profile_mixed:
        return run_profile_mixed(args, cfg)
    if args.profile_ensemble:
        return run_profile_ensemble(args, cfg)
    if args.profile_unet:
        return run_profile_unet(args, cfg)
    if cfg["method"] == "ensemble":
        return run_ensemble(args, cfg)
    if cfg["method"] == "fft-mixed" and not args.profile:
        return run_fft_mixed(args, cfg)
    if cfg["method"] == "learned-mixed" and not args.profile:
        return run_learned_mixed(args, cfg)
    if cfg["method"] == "learned-eval":
        return run_learned_eval(args, cfg)
    return run_plain(args, cfg)


if __name__ == "__main__":
    sys.exit(main())
