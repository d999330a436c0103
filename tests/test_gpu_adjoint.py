"""Adjoint gradients on the GPU against the CPU oracle's discrete adjoint,
against central finite differences of the GPU forward (h = 1e-6), and through
the torch.autograd.Function.

Tolerances: objective vs oracle 1e-12; dJ/dF_n and dJ/du vs the oracle's
adjoint 1e-9 relative to the largest component; finite differences 1e-6
relative (their own truncation/rounding error is ~1e-9..1e-8).
"""
import numpy as np
import pytest

import mpc_tdse
from mpc_tdse.systems import hydrogen_like_1e

pytestmark = pytest.mark.gpu


def _problem(g, seed=0, n_per_l=30, l_max=3, steps=400, K=48):
    s = hydrogen_like_1e(n_per_l, l_max, gauge=g, seed=seed)
    Io, w = mpc_tdse.to_au(2e14, 1.5498)
    tau = mpc_tdse.period(w, 1)
    p = mpc_tdse.pulse_setup("sine", g, Io, w, 0.0, 1, tau)
    rng = np.random.default_rng(seed + 1)
    u = rng.standard_normal(K) * 0.01 * p.Eo
    x0 = np.zeros(s.ntot, complex)
    x0[0] = 1.0
    return s, p, u, steps * 0.1, x0, steps


@pytest.mark.parametrize("path", ["auto", "streaming"])
@pytest.mark.parametrize("g", ["l", "v"])
@pytest.mark.parametrize("target", [-1, 5])
def test_adjoint_matches_oracle(oracle, g, target, path):
    """Both implementations: the persistent resident passes (auto, the
    couplings fit in shared memory) and the streamed step-by-step kernels."""
    s, p, u, T, x0, steps = _problem(g)
    kind = "sineEE" if g == "l" else "sineAA"
    Jo, go, fbo, _ = oracle.objective_gradient(s.n, s.eig, s.dip, g, kind, p.as_array(), u, T,
                                               0.0, 0.1, steps, x0, target)
    with mpc_tdse.Context.from_system(s) as ctx:
        ctx.set_path(path)
        J, gr, fb = ctx.objective_gradient(p, u, T, 0.0, 0.1, steps, x0, target, ckpt_every=64)
    assert abs(J - Jo) < 1e-12
    assert np.max(np.abs(fb - fbo)) <= 1e-9 * np.max(np.abs(fbo))
    assert np.max(np.abs(gr - go)) <= 1e-9 * np.max(np.abs(go))


def test_adjoint_matches_central_differences():
    s, p, u, T, x0, steps = _problem("l", seed=3)
    with mpc_tdse.Context.from_system(s) as ctx:
        J, gr, _ = ctx.objective_gradient(p, u, T, 0.0, 0.1, steps, x0, -1)
        h = 1e-6
        for k in (0, 7, 23, 40):
            up, um = u.copy(), u.copy()
            up[k] += h
            um[k] -= h
            fd = (ctx.objective(p, up, T, 0.0, 0.1, steps, x0) -
                  ctx.objective(p, um, T, 0.0, 0.1, steps, x0)) / (2 * h)
            assert abs(fd - gr[k]) <= 1e-6 * max(abs(fd), 1e-8 * np.max(np.abs(gr))), (k, fd, gr[k])


@pytest.mark.parametrize("path", ["auto", "streaming"])
def test_checkpoint_interval_does_not_change_the_gradient(path):
    s, p, u, T, x0, steps = _problem("v", seed=4, steps=301)
    with mpc_tdse.Context.from_system(s) as ctx:
        ctx.set_path(path)
        J1, g1, f1 = ctx.objective_gradient(p, u, T, 0.0, 0.1, steps, x0, -1, ckpt_every=64)
        J2, g2, f2 = ctx.objective_gradient(p, u, T, 0.0, 0.1, steps, x0, -1, ckpt_every=7)
        J3, g3, f3 = ctx.objective_gradient(p, u, T, 0.0, 0.1, steps, x0, -1, ckpt_every=1000)
    assert J1 == J2 == J3
    assert np.array_equal(g1, g2) and np.array_equal(g1, g3)


def test_objective_equals_plain_forward():
    """The objective's forward pass is the fixed-step propagation itself."""
    s, p, u, T, x0, steps = _problem("l", seed=5)
    with mpc_tdse.Context.from_system(s) as ctx:
        J = ctx.objective(p, np.zeros_like(u), T, 0.0, 0.1, steps, x0, target=-1)
        ct, pop, fld, nrm = ctx.propagate(p, 0.0, 0.1, steps, x0)
    bound = s.eig < 0
    assert abs(J - (1.0 - np.sum(np.abs(ct[bound]) ** 2))) < 1e-13


def test_torch_autograd_function():
    import torch

    from mpc_tdse.autograd import ControlProblem, control_objective

    s, p, u, T, x0, steps = _problem("l", seed=6)
    with mpc_tdse.Context.from_system(s) as ctx:
        prob = ControlProblem(ctx, p, T, 0.0, 0.1, steps, x0)
        ut = torch.tensor(u, dtype=torch.float64, requires_grad=True)
        J = control_objective(ut, prob)
        (2.0 * J).backward()
        J2, g2, _ = ctx.objective_gradient(p, u, T, 0.0, 0.1, steps, x0)
    assert abs(float(J.detach()) - J2) == 0.0
    assert np.allclose(ut.grad.numpy(), 2.0 * g2, rtol=0, atol=1e-15 * np.max(np.abs(g2)) + 1e-300)


@pytest.mark.parametrize("thr", [0.0, -2.0])
def test_2e_ionisation_yields_match_oracle_and_differences(oracle, thr):
    """2e He-CI-like system, velocity gauge: the double-ionisation yield
    (states above the He2+ threshold, thr = 0) and the single-ionisation
    yield (above He+(1s), thr = -2) and their gradients against the oracle's
    adjoint, plus one central difference."""
    from mpc_tdse.systems import helium_like_2e

    s = helium_like_2e((60, 70, 64, 50), gauge="v", seed=3, e_max=8.0)
    Io, w = mpc_tdse.to_au(8e14, 6.2)
    tau = mpc_tdse.period(w, 2)
    p = mpc_tdse.pulse_setup("sine", "v", Io, w, 0.0, 2, tau)
    rng = np.random.default_rng(11)
    K = 64
    u = rng.standard_normal(K) * 0.01 * p.Eo
    x0 = np.zeros(s.ntot, complex)
    x0[0] = 1.0
    steps = int(tau / 0.05)
    oracle.yield_threshold(thr)
    try:
        Jo, go, _, _ = oracle.objective_gradient(s.n, s.eig, s.dip, "v", "sineAA", p.as_array(),
                                                 u, tau, 0.0, 0.05, steps, x0, -1)
    finally:
        oracle.yield_threshold(0.0)
    with mpc_tdse.Context.from_system(s) as ctx:
        ctx.objective_threshold(thr)
        J, gr, _ = ctx.objective_gradient(p, u, tau, 0.0, 0.05, steps, x0, -1)
        h, k = 1e-6, int(np.argmax(np.abs(go)))   # the largest component: FD error ~3e-7
        up, um = u.copy(), u.copy()
        up[k] += h
        um[k] -= h
        fd = (ctx.objective(p, up, tau, 0.0, 0.05, steps, x0) -
              ctx.objective(p, um, tau, 0.0, 0.05, steps, x0)) / (2 * h)
    assert 0.0 < J < 1.0
    assert abs(J - Jo) < 1e-12
    assert np.max(np.abs(gr - go)) <= 1e-9 * np.max(np.abs(go))
    assert abs(fd - gr[k]) <= 1e-6 * max(abs(fd), 1e-8 * np.max(np.abs(gr)))


def test_resident_and_streamed_adjoints_agree():
    s, p, u, T, x0, steps = _problem("l", seed=8, steps=200)
    out = {}
    for path in ("auto", "streaming"):
        with mpc_tdse.Context.from_system(s) as ctx:
            ctx.set_path(path)
            assert ctx.path == ("resident" if path == "auto" else "streaming")
            out[path] = ctx.objective_gradient(p, u, T, 0.0, 0.1, steps, x0, -1, ckpt_every=16)
    (J1, g1, f1), (J2, g2, f2) = out["auto"], out["streaming"]
    assert abs(J1 - J2) < 1e-14
    assert np.max(np.abs(g1 - g2)) <= 1e-12 * np.max(np.abs(g2))
    assert np.max(np.abs(f1 - f2)) <= 1e-12 * np.max(np.abs(f2))


@pytest.mark.parametrize("g", ["l", "v"])
@pytest.mark.parametrize("steps,ckpt", [(301, 64), (128, 64), (50, 64), (37, 1)])
def test_fused_reverse_pass_equals_per_segment_passes(g, steps, ckpt, monkeypatch):
    """The fused reverse pass (each segment's recompute concurrent with the
    next segment's sweep, one persistent launch) against the per-segment
    resident launches (recompute, then sweep): the same arithmetic per row
    and the same reduction orders, so the same gradient; segment counts from
    1 to many, a short last segment, one-step segments."""
    s, p, u, T, x0, _ = _problem(g, seed=9, steps=steps)
    out = []
    for fused in (True, False):
        if not fused:
            monkeypatch.setenv("MPC_NO_FUSED_ADJOINT", "1")
        with mpc_tdse.Context.from_system(s) as ctx:
            assert ctx.path == "resident"
            out.append(ctx.objective_gradient(p, u, T, 0.0, 0.1, steps, x0, -1, ckpt))
    (J1, g1, f1), (J2, g2, f2) = out
    assert J1 == J2
    assert np.max(np.abs(g1 - g2)) <= 1e-13 * np.max(np.abs(g2))
    assert np.max(np.abs(f1 - f2)) <= 1e-13 * np.max(np.abs(f2))


def test_mpc_adjoint_is_the_objective_gradient():
    """mpc_adjoint (one call from controls to gradient) returns exactly what
    mpc_objective_gradient returns."""
    import ctypes as C

    s, p, u, T, x0, steps = _problem("v", seed=3, steps=120)
    L = mpc_tdse.lib()
    xs = x0.astype(np.complex128).view(np.float64).copy()
    out = []
    with mpc_tdse.Context.from_system(s) as ctx:
        for fn in (L.mpc_objective_gradient, L.mpc_adjoint):
            J = np.zeros(1)
            g = np.zeros(len(u))
            f = np.zeros(steps)
            dp = C.POINTER(C.c_double)
            rc = fn(ctx._h, C.byref(p), len(u), u.ctypes.data_as(dp), T, 0.0, 0.1, steps, -1, 32,
                    xs.ctypes.data_as(dp), J.ctypes.data_as(dp), g.ctypes.data_as(dp),
                    f.ctypes.data_as(dp))
            assert rc == 0, mpc_tdse.last_error()
            out.append((J, g, f))
    for a, b in zip(*out):
        assert np.array_equal(a, b)
