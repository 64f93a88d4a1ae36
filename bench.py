#!/usr/bin/env python
"""Benchmark of the mobydiff RK3 time step on B200.

Workload (default ``--config c1``): the wavy-wall channel with immersed
boundary on a 256x128x128 staggered grid, FP64, Re 3000, dt 1e-3, red-black
SOR (omega 1.7) to residual 1e-10, walls y = y0 + A sin(2 pi x / lambda)
(and +2) with A = 0.05, lambda = Lx/2, seeded Poiseuille + noise initial
condition projected at t = 0.  One step = one full RK3 step (3 predictor
passes, 3 projections to tolerance, boundary conditions).

Prints ONE JSON line on rank 0.  ``value`` is Mcell-steps/s with fields
resident in HBM; ``e2e`` is the same metric through the C ABI with the
state copied host->device and device->host (pinned buffers) every step.
``--impl reference`` times the CPU restatement of the reference (the
oracle) on the host cores instead.

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

CONFIGS = {
    "c1": dict(workload="wavy-wall IBM channel 256x128x128, FP64 red-black SOR omega=1.7 to residual 1e-10",
               nx=256, ny=128, nz=128, lx=2 * math.pi, ly=2.25, lz=math.pi, re=3000.0, dt=1e-3,
               solver="redblack", sor=1.7, tol=1e-10, check_every=50, ibm="wavy", amp=0.05),
    "c0": dict(workload="periodic channel 64^3, FP64 FFT+Thomas", nx=64, ny=64, nz=64, lx=2 * math.pi, ly=2.0,
               lz=math.pi, re=2000.0, dt=1e-3, solver="fft", ibm="none", amp=0.0),
    "c2": dict(workload="periodic channel 512x256x256, FP64 FFT+Thomas", nx=512, ny=256, nz=256,
               lx=4 * math.pi, ly=2.0, lz=2 * math.pi, re=5000.0, dt=1e-3, solver="fft", ibm="none", amp=0.0),
}

# Red-black iterations per RK3 step of the c1 workload in the steps the
# default run times (warm-up 3, steps 3), measured on B200; the oracle's
# sweeps are bit-identical, so its iteration count is the same.  Used only
# to scale the reference arm's bounded CPU sample to a full step.
C1_ITERS_PER_STEP = 48000.0

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


def _setup(cfg, M, device, profile=False):
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
        opts = M.make_solver_opts(M.SOLVER_REDBLACK, sor=cfg["sor"], n_iter=20, tol=0.0)
    elif cfg["solver"] == "redblack":
        opts = M.make_solver_opts(M.SOLVER_REDBLACK, sor=cfg["sor"], tol=cfg["tol"], check_every=cfg["check_every"],
                                  max_iter=200000)
    else:
        opts = M.make_solver_opts(M.SOLVER_FFT)
    s.init_pressure_solver(opts)
    s.channel_ic(SEED, 0.1, 0.01, y0, cfg["amp"], lam)
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


def run_reference(args, cfg):
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    iters = C1_ITERS_PER_STEP if cfg["solver"] == "redblack" else 0.0
    vals = []
    for step in range(args.warmup + args.steps):
        ph, cells = _oracle_sample(cfg, threads, target_s=6.0)
        if step >= args.warmup:
            vals.append(cells / _cpu_step_seconds(cfg, ph, iters) / 1e6)
    value = float(np.median(vals))
    if cfg["solver"] == "redblack":
        sample = (f"per step: 3 predictor passes + ~{ph['sor_iters_sampled']} red-black iterations of the "
                  f"{int(iters)} a full step needs, on the full {cfg['nx']}x{cfg['ny']}x{cfg['nz']} grid; "
                  "step time extrapolated by iteration count")
    else:
        sample = "one full RK3 step on the full grid"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": cfg["workload"], "arm": "CPU restatement of the reference (oracle), OpenMP"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, cfg):
    import torch
    import mobydiff_b200 as M

    ws, rank, local = _dist()
    device = local
    torch.cuda.set_device(device)
    pg = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900),
                                device_id=torch.device("cuda", device))
        pg = dist

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
    # The state at the start of the timed steps, kept on the host so that the
    # end-to-end leg below replays exactly the same steps (same iteration
    # counts).  At a step boundary u, v, w, p are the whole state: beta_1 = 0
    # (step.f90:22), so oldrhs is not read before it is rewritten.
    host = None
    if not args.no_e2e:
        host = [torch.empty(s.padded, dtype=torch.float64, pin_memory=True) for _ in range(4)]
        s.update_host(*[h.numpy() for h in host])

    # ---- timed region: device-resident state --------------------------------
    s.set_timing(True)
    clocks = ClockSampler(device)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    clocks.start()
    launches0 = s.launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    iters = 0
    for _ in range(args.steps):
        iters += s.step(1)
    ev1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    if pg:
        pg.barrier()
    launches = s.launch_count() - launches0
    ms = ev0.elapsed_time(ev1)
    tim = s.get_timing()
    s.set_timing(False)
    ms_all = ms
    if pg:
        t = torch.tensor([ms], device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms_all = float(t.item())
    value = ws * cells * args.steps / (ms_all / 1e3) / 1e6

    # ---- end to end through the C ABI with host buffers -------------------
    # every step: the state (u, v, w, p) host->device from pinned memory,
    # one RK3 step, the state device->host
    e2e_line = None
    if not args.no_e2e:
        nbytes = 4 * host[0].numel() * 8
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        e2e_iters = 0
        for _ in range(args.steps):
            s.update_device(*[h.numpy() for h in host])
            e2e_iters += s.step(1)
            s.update_host(*[h.numpy() for h in host])
        e1.record(stream)
        torch.cuda.synchronize()
        ems = e0.elapsed_time(e1)
        if pg:
            t = torch.tensor([ems], device="cuda")
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            ems = float(t.item())
        e2e = ws * cells * args.steps / (ems / 1e3) / 1e6
        e2e_line = {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
                    "same_steps_as_value": e2e_iters == iters}

    # ---- roofline of the dominant kernel ------------------------------------
    peak, peak_kind = _peaks()
    if cfg["solver"] == "redblack":
        kname, alg_per_cell = "sor_sweep", 32.0          # 4 doubles per cell per colour sweep
    else:
        kname, alg_per_cell = "momentum", 112.0          # 14 doubles per cell
    kms, kn = tim[kname]
    avg_s = (kms / 1e3) / max(kn, 1)
    alg_bytes = alg_per_cell * cells
    achieved = alg_bytes / avg_s / 1e9 if kn else None
    tpc = _traffic_per_cell(kname)
    share = kms / ms if ms > 0 else None
    roofline = {"kernel": kname, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None, "peak_kind": peak_kind,
                "traffic": (tpc * cells) if tpc else None, "algorithmic_bytes": alg_bytes,
                "avg_launch_ms": avg_s * 1e3, "launches": kn, "share_of_step_time": share}

    iters_per_substage = iters / (3 * args.steps) if cfg["solver"] == "redblack" else 0
    sor_kernel = None
    if cfg["solver"] == "redblack":
        names = {1: "one launch per colour sweep", 2: "fused red+black pass 32x8", 3: "fused red+black pass 32x16"}
        sor_kernel = names.get(s.last_solve_stats().variant, "?")

    # ---- CPU baseline (rank 0, one GPU only) -------------------------------
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        ph, _ = _oracle_sample(cfg, threads)
        per_step = _cpu_step_seconds(cfg, ph, iters / max(args.steps, 1))
        if cfg["solver"] == "redblack":
            sample = (f"3 predictor passes + {ph['sor_iters_sampled']} red-black iterations on the full grid; "
                      f"step time extrapolated to the {iters / max(args.steps, 1):.0f} iterations per step of "
                      "the timed GPU steps (the sweeps are bit-identical, so are the counts)")
        else:
            sample = "one predictor + one FFT projection on the full grid, x3 substages"
        cpu = {"value": cells / per_step / 1e6, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_all / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic: seeded Poiseuille+noise IC (SplitMix64), projected at t=0",
                "config": {"workload": cfg["workload"], "grid": [cfg["nx"], cfg["ny"], cfg["nz"]],
                           "re": cfg["re"], "dt": cfg["dt"], "method": "plain FP64",
                           "parallelism": f"replicas x{ws}",
                           "l2": "inputs larger than L2 (state + IBM coefficients > 126 MB)"},
                "poisson_iters_per_substage": iters_per_substage,
                "sor_kernel": sor_kernel,
                "roofline": roofline, "cpu_baseline": cpu, "clocks": clk,
                "e2e": e2e_line, "gpu_launches": launches}
        print(json.dumps(line), flush=True)
    s.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c1", choices=sorted(CONFIGS))
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg")
    ap.add_argument("--profile", action="store_true",
                    help="profiling run for ncu: full-size state, fixed 20 red-black iterations per projection")
    args = ap.parse_args()
    cfg = CONFIGS[args.config]
    if args.impl == "reference":
        return run_reference(args, cfg)
    return run_ours(args, cfg)


if __name__ == "__main__":
    sys.exit(main())
