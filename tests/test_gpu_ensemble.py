"""Batched ensemble: every member against the single-context path run
alone (bit for bit with a fixed iteration count), CUDA-graph replay against
eager launches, and the autotuner's cache."""
import json

import numpy as np
import pytest

import mobydiff_b200 as M
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu

MEMBERS = [
    dict(nx=32, ny=32, nz=32, re=3000.0, amp=0.05, seed=11),
    dict(nx=48, ny=32, nz=64, re=1500.0, amp=0.08, seed=12),
    dict(nx=64, ny=48, nz=32, re=4200.0, amp=0.0, seed=13),
]


def _members():
    return [M.make_member(**m) for m in MEMBERS]


def _single(m, opts, mode):
    g = M.make_grid(m.nx, m.ny, m.nz, m.lx, m.ly, m.lz, m.re, m.dt, (2.0 / m.re, 0.0, 0.0))
    s = M.Solver(g, M.channel_bc(), 0)
    s.enter_field_data()
    y0 = (m.ly - 2.0) / 2.0
    lam = m.lx / 2.0
    if m.amp > 0.0:   # the ensemble generates its members' coefficients on the device too
        s.enter_ibm_geometry(M.ibm_wavy(m.amp, lam, y0))
    s.init_pressure_solver(opts)
    s.set_pressure_guess(mode, record=mode != M.GUESS_ZERO)
    s.channel_ic(m.seed, 0.1, 0.01, y0, m.amp, lam)
    return s


@pytest.mark.parametrize("mode", [M.GUESS_ZERO, M.GUESS_EXTRAPOLATED])
def test_fixed_iterations_bitwise_equal_to_single_channels(mode):
    opts = M.make_solver_opts(M.SOLVER_REDBLACK, sor=1.7, n_iter=30, tol=0.0)
    mems = _members()
    with M.Ensemble(mems, opts) as E:
        E.set_guess(mode)
        E.ic()
        for q, m in enumerate(mems):   # the t=0 projection alone
            with _single(m, opts, mode) as s:
                for n in ("un", "vn", "wn", "pn"):
                    assert np.array_equal(E.get(q, n), s.get(n)), (q, n)
        E.step(3)
        for q, m in enumerate(mems):
            with _single(m, opts, mode) as s:
                s.step(3)
                for n in ("un", "vn", "wn", "pn"):
                    assert np.array_equal(E.get(q, n), s.get(n)), (q, n)
                st, tot = E.member_stats(q)
                assert st.iterations == 30 and tot == 9 * 30


def test_tolerance_mode_matches_single_channels():
    # the ensemble checks every check_every iterations: the single channels too
    opts = M.make_solver_opts(M.SOLVER_REDBLACK, sor=1.7, tol=1e-8, check_every=10, max_iter=200000,
                              adaptive_checks=False)
    mems = _members()
    with M.Ensemble(mems, opts) as E:
        E.set_guess(M.GUESS_EXTRAPOLATED)
        E.ic()
        it_e = E.step(4)
        it_s = 0
        for q, m in enumerate(mems):
            with _single(m, opts, M.GUESS_EXTRAPOLATED) as s:
                it_s += s.step(4)
                st, _ = E.member_stats(q)
                ss = s.last_solve_stats()
                assert st.status == 0 and abs(st.iterations - ss.iterations) <= 10, (q, st.iterations, ss.iterations)
                assert st.residual <= 1e-8 * 1.0000001 or st.residual * st.residual0 <= st.atol * 1.0000001
                for n in ("un", "vn", "wn"):
                    assert rel_l2(E.get(q, n), s.get(n)) <= 1e-6, (q, n)
        print("iterations: ensemble", it_e, "single channels", it_s)
        assert abs(it_e - it_s) <= 0.02 * it_s + 30 * len(mems)


def test_graph_replay_equals_eager_launches():
    opts = M.make_solver_opts(M.SOLVER_REDBLACK, sor=1.7, tol=1e-8, check_every=10, max_iter=200000)
    mems = _members()
    with M.Ensemble(mems, opts) as A, M.Ensemble(mems, opts) as B:
        for E in (A, B):
            E.set_guess(M.GUESS_EXTRAPOLATED)
            E.ic()
        B.use_graph(False)
        ia, ib = A.step(3), B.step(3)
        assert ia == ib
        print("graph:", A.info())
        assert not B.info()["graph"]
        for q in range(len(mems)):
            for n in ("un", "vn", "wn", "pn"):
                assert np.array_equal(A.get(q, n), B.get(q, n)), (q, n)


def test_autotuner_choice_is_cached_and_results_unchanged(tmp_path):
    cache = str(tmp_path / "ensemble_tune.json")
    opts = M.make_solver_opts(M.SOLVER_REDBLACK, sor=1.7, n_iter=20, tol=0.0)
    mems = _members()
    with M.Ensemble(mems, opts) as A, M.Ensemble(mems, opts) as B:
        for E in (A, B):
            E.set_guess(M.GUESS_EXTRAPOLATED)
            E.ic()
        t, b, lr, ms = A.tune(cache)
        assert t in (128, 256, 512) and b in (1, 2, 4, 8) and ms > 0.0
        data = json.load(open(cache))
        entry = list(data.values())[0]
        assert len(data) == 1 and entry["threads"] == t and entry["low_regs"] == int(lr)
        assert B.tune(cache) == (t, b, lr, -1.0)   # cache hit: no timing
        B.config(128, 1, low_regs=not lr)
        A.step(2)
        B.step(2)
        for q in range(len(mems)):
            for n in ("un", "vn", "wn", "pn"):
                assert np.array_equal(A.get(q, n), B.get(q, n)), (q, n)


def test_ensemble_argument_checks():
    opts = M.make_solver_opts(M.SOLVER_REDBLACK, sor=1.7, n_iter=5, tol=0.0)
    with pytest.raises(M.MdxError):
        M.Ensemble([M.make_member(33, 16, 16)], opts)   # odd nx
    with pytest.raises(M.MdxError):
        M.Ensemble([M.make_member(32, 16, 16)], M.make_solver_opts(M.SOLVER_FFT))
    with M.Ensemble([M.make_member(32, 16, 16)], opts) as E:
        with pytest.raises(M.MdxError):
            E.config(100)
        with pytest.raises(M.MdxError):
            E.set_guess(M.GUESS_LEARNED)


def test_mixed_precision_members_match_single_channels():
    """FP32 sweeps in FP64 defect correction inside the persistent kernel:
    each member lands within the solve tolerance of the single-context mixed
    path and of the FP64 ensemble (the FP32 arithmetic is not bit-equal: the
    ensemble file is built without FMA contraction)."""
    # the ensemble's FP32 sweeps are the face form: the single contexts run it too
    mix = M.make_solver_opts(M.SOLVER_REDBLACK, sor=1.7, tol=1e-8, check_every=10, max_iter=200000,
                             precision=M.PREC_MIXED, inner_form=1)
    f64 = M.make_solver_opts(M.SOLVER_REDBLACK, sor=1.7, tol=1e-8, check_every=10, max_iter=200000)
    mems = _members()
    with M.Ensemble(mems, mix) as E, M.Ensemble(mems, f64) as F:
        for X in (E, F):
            X.set_guess(M.GUESS_EXTRAPOLATED)
            X.ic()
        ie, i_f = E.step(4), F.step(4)
        print("iterations: ensemble mixed", ie, "ensemble fp64", i_f)
        for q, m in enumerate(mems):
            st, _ = E.member_stats(q)
            assert st.status == 0 and st.variant > 100
            assert st.residual <= 1e-8 * 1.0000001 or st.residual * st.residual0 <= st.atol * 1.0000001
            with _single(m, mix, M.GUESS_EXTRAPOLATED) as s:
                s.step(4)
                for other in (s.get, lambda n: F.get(q, n)):
                    num = sum(float(np.sum((E.get(q, n) - other(n)) ** 2)) for n in ("un", "vn", "wn"))
                    den = sum(float(np.sum(other(n) ** 2)) for n in ("un", "vn", "wn"))
                    assert (num / den) ** 0.5 <= 1e-6, q          # the velocity vector
                    for n in ("un", "vn", "wn"):                  # each component, v and w of small norm
                        assert rel_l2(E.get(q, n), other(n)) <= 1e-5, (q, n)


def test_potential_form_members_match_single_channels():
    """The potential form of the FP32 sweeps inside the persistent kernel
    (each cell's phi in place of the face corrections): every member meets
    the tolerance and lands within the solve tolerance of the single-context
    potential form and of the face-form ensemble (velocity vector 1e-6, each
    component 1e-5)."""
    # inner_form 2: the potential form in the ensemble's kernel too (its default is the face form)
    pot = M.make_solver_opts(M.SOLVER_REDBLACK, sor=1.7, tol=1e-8, check_every=10, max_iter=200000,
                             precision=M.PREC_MIXED, inner_form=2)
    face = M.make_solver_opts(M.SOLVER_REDBLACK, sor=1.7, tol=1e-8, check_every=10, max_iter=200000,
                              precision=M.PREC_MIXED, inner_form=1)
    mems = _members()
    with M.Ensemble(mems, pot) as E, M.Ensemble(mems, face) as F:
        for X in (E, F):
            X.set_guess(M.GUESS_EXTRAPOLATED)
            X.ic()
        ie, i_f = E.step(4), F.step(4)
        print("iterations: potential", ie, "face", i_f)
        assert ie <= 1.3 * i_f + 100
        for q, m in enumerate(mems):
            st, _ = E.member_stats(q)
            assert st.status == 0 and st.variant // 100 == 7, (q, st.variant)
            assert st.residual <= 1e-8 * 1.0000001 or st.residual * st.residual0 <= st.atol * 1.0000001
            with _single(m, pot, M.GUESS_EXTRAPOLATED) as s:
                s.step(4)
                for other in (s.get, lambda n: F.get(q, n)):
                    num = sum(float(np.sum((E.get(q, n) - other(n)) ** 2)) for n in ("un", "vn", "wn"))
                    den = sum(float(np.sum(other(n) ** 2)) for n in ("un", "vn", "wn"))
                    assert (num / den) ** 0.5 <= 1e-6, q
                    for n in ("un", "vn", "wn"):
                        assert rel_l2(E.get(q, n), other(n)) <= 1e-5, (q, n)


def test_sixteen_uneven_members_bitwise_and_mixed():
    """16 members of uneven sizes drawn like the 64-member configuration (nx,
    nz in 32..128, ny in 32..96, multiples of 16; Re in 1000..5000; A in
    0..0.1): with a fixed iteration count every member equals its single
    context bit for bit; with FP32 sweeps in FP64 defect correction to 1e-8
    every member's velocity is within 1e-6 of its single context."""
    import bench
    mems = bench.ensemble_members(M, 16, seed=20261207)
    sizes = {(m.nx, m.ny, m.nz) for m in mems}
    assert len(sizes) >= 10
    opts = M.make_solver_opts(M.SOLVER_REDBLACK, sor=1.7, n_iter=20, tol=0.0)
    with M.Ensemble(mems, opts) as E:
        E.set_guess(M.GUESS_EXTRAPOLATED)
        E.ic()
        E.step(2)
        for q, m in enumerate(mems):
            with _single(m, opts, M.GUESS_EXTRAPOLATED) as s:
                s.step(2)
                for n in ("un", "vn", "wn", "pn"):
                    assert np.array_equal(E.get(q, n), s.get(n)), (q, n)
    # the ensemble's FP32 sweeps are the face form: the single contexts run it too
    opts = M.make_solver_opts(M.SOLVER_REDBLACK, sor=1.7, tol=1e-8, check_every=10, max_iter=200000,
                              precision=M.PREC_MIXED, adaptive_checks=False, inner_form=1)
    with M.Ensemble(mems, opts) as E:
        E.set_guess(M.GUESS_EXTRAPOLATED)
        E.ic()
        E.step(2)
        for q, m in enumerate(mems):
            with _single(m, opts, M.GUESS_EXTRAPOLATED) as s:
                s.step(2)
                st, _ = E.member_stats(q)
                assert st.status == 0, q
                for n in ("un", "vn", "wn"):
                    assert rel_l2(E.get(q, n), s.get(n)) <= 1e-6, (q, n)


def test_learned_warm_start_in_the_ensemble():
    """The learned warm start inside the ensemble: a network trained on one
    context's snapshots (fully convolutional, so it applies to every member's
    grid) is loaded into a 4-member ensemble of uneven sizes; with FP32 sweeps
    in FP64 defect correction to 1e-8 the members converge, the network's
    corrections are applied (kept or undone by the divergence test) and every
    member's velocity agrees with the same ensemble started from the
    extrapolated increment alone within 1e-6; the step stays one CUDA graph."""
    from mobydiff_b200 import learned
    s, g = learned.wavy_solver(32, 32, 32, 3000.0, 0.05, 1e-8, check_every=10, precision=M.PREC_MIXED)
    with s:
        net = learned.record_and_train(s, g, [(31, 0.03, 2000.0), (32, 0.07, 4000.0)], warm_steps=3, record_steps=3,
                                       iters=200, channels=32)
    mems = [M.make_member(nx=32, ny=32, nz=32, re=2500.0, amp=0.05, seed=41),
            M.make_member(nx=64, ny=48, nz=32, re=3500.0, amp=0.08, seed=42),
            M.make_member(nx=48, ny=32, nz=64, re=1500.0, amp=0.02, seed=43),
            M.make_member(nx=32, ny=64, nz=48, re=4500.0, amp=0.0, seed=44)]
    opts = M.make_solver_opts(M.SOLVER_REDBLACK, sor=1.7, tol=1e-8, check_every=10, max_iter=200000,
                              precision=M.PREC_MIXED, adaptive_checks=False)
    out = {}
    for mode in (M.GUESS_EXTRAPOLATED, M.GUESS_LEARNED, "gated"):
        with M.Ensemble(mems, opts) as E:
            if mode == M.GUESS_LEARNED:
                E.unet_load(net.params, net.out_scale, channels=net.channels)
            if mode == "gated":   # the correction per member and substage only while it saves iterations
                E.unet_load(net.params, net.out_scale, channels=net.channels, gate_period=4)
                mode = M.GUESS_LEARNED
                key = "gated"
            else:
                key = mode
            E.set_guess(mode)
            E.ic()
            its = E.step(6)
            for q in range(len(mems)):
                st, _ = E.member_stats(q)
                assert st.status == 0, (mode, q)
            out[key] = (its, [E.get(q, "un") for q in range(len(mems))], [E.get(q, "vn") for q in range(len(mems))],
                        E.unet_stats() if mode == M.GUESS_LEARNED else None, E.info())
    its_l, u_l, v_l, (kept, undone, gated), info = out[M.GUESS_LEARNED]
    its_x, u_x, v_x, _, _ = out[M.GUESS_EXTRAPOLATED]
    its_g, u_g, _, (kept_g, undone_g, gated_g), _ = out["gated"]
    print("iterations extrapolated", its_x, "learned", its_l, "corrections kept", kept, "undone", undone,
          "graph", info["graph"], "gated: iterations", its_g, "kept", kept_g, "undone", undone_g, "left", gated_g)
    assert kept + undone > 0 and gated == 0
    assert gated_g > 0 and kept_g + undone_g > 0
    for q in range(len(mems)):
        assert rel_l2(u_g[q], u_x[q]) <= 1e-6, q
    for q in range(len(mems)):
        assert rel_l2(u_l[q], u_x[q]) <= 1e-6, q
    assert info["graph"]
