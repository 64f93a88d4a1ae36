"""Training pipeline of the learned warm start: run the solver on a few
seeded wavy-channel cases, record snapshots of its projections on the
device, and train the network there.

The solver records a snapshot in every converged red-black projection that
starts from the extrapolated increment (guess mode EXTRAPOLATED or
LEARNED): the divergence that guess leaves, the two previous increments and
the IBM factor as inputs, the rest of the converged increment as target
(include/mobydiff_b200.h, "learned warm start").  Training is Adam on one
snapshot per step, a seeded random order, on the device.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import (GUESS_EXTRAPOLATED, SOLVER_REDBLACK, PREC_FP64, Solver, channel_bc, ibm_wavy, make_grid,
               make_solver_opts, set_ibm_coeff)


@dataclass
class TrainedNet:
    params: np.ndarray
    out_scale: float
    channels: int
    extra_bottleneck: int
    slope: float
    loss_first: float
    loss_last: float
    snapshots: int
    record_seconds: float
    train_ms: float
    runs: list = field(default_factory=list)


def wavy_solver(nx, ny, nz, re, amp, tol, check_every=50, precision=PREC_FP64, device=0, ly=2.25,
                lx=2 * math.pi, lz=math.pi, dt=1e-3):
    """A wavy-wall IBM channel (walls at y0 + A sin(2 pi x / (Lx/2)) and
    y0 + 2 + ..., y0 = (Ly - 2)/2) with the red-black projection; no IC yet."""
    g = make_grid(nx, ny, nz, lx, ly, lz, re, dt, (2.0 / re, 0.0, 0.0))
    s = Solver(g, channel_bc(), device)
    s.enter_field_data()
    y0 = (ly - 2.0) / 2.0
    if amp > 0.0:
        s.enter_ibm_data(*set_ibm_coeff(g, ibm_wavy(amp, lx / 2, y0)))
    s.init_pressure_solver(make_solver_opts(SOLVER_REDBLACK, sor=1.7, tol=tol, check_every=check_every,
                                            max_iter=400000, precision=precision))
    return s, g


def record_and_train(s: Solver, g, runs, warm_steps: int = 3, record_steps: int = 8, iters: int = 600,
                     lr: float = 3e-4, channels: int = 32, extra_bottleneck: int = 0, slope: float = 0.1,
                     seed: int = 20261203) -> TrainedNet:
    """Record snapshots on `s` for each (seed, amplitude) or (seed, amplitude,
    Re) in `runs` -- a fresh channel IC each, `warm_steps` steps to build the
    increment history, then `record_steps` recorded steps (three snapshots
    each) -- and train.

    The IBM coefficients of `s` are replaced per run (generated on the
    device), and Re with its body force 2/Re when a run gives one; the grid is
    the solver's.  The first half of the Adam steps runs at lr, the second at
    lr/3.
    """
    ly = g.ly
    y0 = (ly - 2.0) / 2.0
    lam = g.lx / 2.0
    cap = 3 * record_steps * len(runs)
    s.unet_create(channels=channels, extra_bottleneck=extra_bottleneck, capacity=cap, slope=slope, seed=seed)
    s.set_pressure_guess(GUESS_EXTRAPOLATED, record=True)
    t0 = time.time()
    for run in runs:
        run_seed, amp = run[0], run[1]
        if len(run) > 2:
            s.set_flow(run[2])
        if amp > 0.0:
            s.enter_ibm_geometry(ibm_wavy(amp, lam, y0))
        else:
            s.exit_ibm_data()
        s.unet_record(False)
        s.channel_ic(run_seed, 0.1, 0.01, y0, amp, lam)
        s.step(warm_steps)
        s.unet_record(True)
        s.step(record_steps)
    s.unet_record(False)
    rec = time.time() - t0
    l0, _ = s.unet_train(iters // 2, lr)
    tm = s.unet_stats().train_ms
    _, l1 = s.unet_train(iters - iters // 2, lr / 3.0)
    st = s.unet_stats()
    return TrainedNet(params=s.unet_params(), out_scale=s.unet_out_scale(), channels=channels,
                      extra_bottleneck=extra_bottleneck, slope=slope, loss_first=l0, loss_last=l1,
                      snapshots=int(st.snapshots), record_seconds=rec, train_ms=tm + st.train_ms, runs=list(runs))


def load_into(s: Solver, net: TrainedNet, step_rule: int = 0, gate_period: int = 0) -> None:
    """Give solver `s` (same grid) the trained network, without snapshot
    storage; step_rule 1 scales each correction by its energy-optimal step;
    gate_period > 0 applies the correction per RK substage only while it
    takes fewer iterations than the extrapolated guess alone."""
    s.unet_create(channels=net.channels, extra_bottleneck=net.extra_bottleneck, capacity=0, slope=net.slope,
                  step_rule=step_rule, gate_period=gate_period)
    s.unet_set_params(net.params)
    s.unet_out_scale(net.out_scale)
