"""Batched objective and gradient (many pulses through the FP64 tensor-core
stage GEMM) against the single-pulse GPU adjoint, the CPU oracle's adjoint
and central differences.

Tolerances: objectives 1e-12 absolute (1e-13 relative for small yields); dJ/du
and dJ/dF_n 1e-9 relative to the largest component (the GEMM sums the
coupling in another order than the streamed single-pulse kernel and the
oracle's loops); central differences 1e-6 relative.
"""
import numpy as np
import pytest

import mpc_tdse
from mpc_tdse.systems import helium_like_2e, hydrogen_like_1e

pytestmark = pytest.mark.gpu


def _pulses(g, specs):
    out = []
    for Io_W, w_eV, cyc, cep in specs:
        Io, w = mpc_tdse.to_au(Io_W, w_eV)
        tau = mpc_tdse.period(w, cyc)
        out.append((mpc_tdse.pulse_setup("sine", g, Io, w, cep, cyc, tau), tau))
    return out


def _batch(g, B=5, K=40, seed=0):
    rng = np.random.default_rng(seed)
    specs = [(10 ** rng.uniform(13.5, 14.5), rng.uniform(1.4, 3.0), 1, 0.0) for _ in range(B)]
    ps = _pulses(g, specs)
    U = np.stack([rng.standard_normal(K) * 0.01 * p.Eo for p, _ in ps])
    T = np.array([tau for _, tau in ps])
    return [p for p, _ in ps], U, T


@pytest.mark.parametrize("g", ["l", "v"])
@pytest.mark.parametrize("target", [-1, 4])
def test_batch_gradient_matches_single_pulse_adjoint(g, target):
    s = hydrogen_like_1e(36, 3, gauge=g, seed=1)
    pulses, U, T = _batch(g)
    B = len(pulses)
    steps = 300
    X0 = np.zeros((B, s.ntot), complex)
    X0[:, 0] = 1.0
    with mpc_tdse.Context.from_system(s) as ctx:
        J, G, Fb = ctx.batch_objective_gradient(pulses, U, T, 0.0, 0.1, steps, X0, target,
                                                ckpt_every=32)
        for b in range(B):
            j1, g1, f1 = ctx.objective_gradient(pulses[b], U[b], T[b], 0.0, 0.1, steps, X0[b],
                                                target, ckpt_every=32)
            assert abs(J[b] - j1) < 1e-12, b
            assert np.max(np.abs(G[b] - g1)) <= 1e-9 * np.max(np.abs(g1)), b
            assert np.max(np.abs(Fb[b] - f1)) <= 1e-9 * np.max(np.abs(f1)), b


def test_batch_gradient_matches_oracle(oracle):
    s = hydrogen_like_1e(30, 3, gauge="l", seed=2)
    pulses, U, T = _batch("l", B=3, K=48, seed=5)
    steps = 250
    X0 = np.zeros((3, s.ntot), complex)
    X0[:, 0] = 1.0
    with mpc_tdse.Context.from_system(s) as ctx:
        J, G, _ = ctx.batch_objective_gradient(pulses, U, T, 0.0, 0.1, steps, X0, -1)
    for b in range(3):
        Jo, go, _, _ = oracle.objective_gradient(s.n, s.eig, s.dip, "l", "sineEE",
                                                 pulses[b].as_array(), U[b], T[b], 0.0, 0.1,
                                                 steps, X0[b], -1)
        assert abs(J[b] - Jo) < 1e-12
        assert np.max(np.abs(G[b] - go)) <= 1e-9 * np.max(np.abs(go))


@pytest.mark.parametrize("thr", [0.0, -2.0])
def test_batch_2e_yields_and_central_difference(thr):
    """Double (thr = 0) and single (thr = -2) ionisation yields of a 2e
    He-like system for 4 pulses; one central difference per pulse."""
    s = helium_like_2e((40, 48, 44, 36), gauge="v", seed=4, e_max=8.0)
    rng = np.random.default_rng(7)
    specs = [(10 ** rng.uniform(14.5, 15), rng.uniform(5.0, 7.0), 2, 0.0) for _ in range(4)]
    ps = _pulses("v", specs)
    pulses = [p for p, _ in ps]
    K = 32
    U = np.stack([rng.standard_normal(K) * 0.01 * p.Eo for p in pulses])
    T = np.array([tau for _, tau in ps])
    steps = int(max(T) / 0.05) + 1
    X0 = np.zeros((4, s.ntot), complex)
    X0[:, 0] = 1.0
    with mpc_tdse.Context.from_system(s) as ctx:
        ctx.objective_threshold(thr)
        J, G, _ = ctx.batch_objective_gradient(pulses, U, T, 0.0, 0.05, steps, X0, -1)
        for b in range(4):
            j1, g1, _ = ctx.objective_gradient(pulses[b], U[b], T[b], 0.0, 0.05, steps, X0[b], -1)
            assert abs(J[b] - j1) <= 1e-13 * max(j1, 1e-300) + 1e-16, b
            assert np.max(np.abs(G[b] - g1)) <= 1e-9 * np.max(np.abs(g1)), b
        h = 1e-6
        k = [int(np.argmax(np.abs(G[b]))) for b in range(4)]
        Up, Um = U.copy(), U.copy()
        for b in range(4):
            Up[b, k[b]] += h
            Um[b, k[b]] -= h
        Jp = ctx.batch_objective(pulses, Up, T, 0.0, 0.05, steps, X0, -1)
        Jm = ctx.batch_objective(pulses, Um, T, 0.0, 0.05, steps, X0, -1)
    for b in range(4):
        fd = (Jp[b] - Jm[b]) / (2 * h)
        assert 0.0 < J[b] < 1.0
        assert abs(fd - G[b, k[b]]) <= 1e-6 * abs(fd), (b, fd, G[b, k[b]])


def test_batch_checkpoint_interval_is_bit_identical():
    s = hydrogen_like_1e(32, 3, gauge="v", seed=3)
    pulses, U, T = _batch("v", B=6, K=24, seed=9)
    X0 = np.zeros((6, s.ntot), complex)
    X0[:, 0] = 1.0
    with mpc_tdse.Context.from_system(s) as ctx:
        r = [ctx.batch_objective_gradient(pulses, U, T, 0.0, 0.1, 201, X0, -1, ckpt_every=c)
             for c in (64, 9, 500, 0)]   # 0: sized to free memory (one segment here)
    for J, G, Fb in r[1:]:
        assert np.array_equal(J, r[0][0]) and np.array_equal(G, r[0][1])
        assert np.array_equal(Fb, r[0][2])


def test_batch_objective_after_reallocation_is_bit_identical():
    """Work buffers re-sized between calls (checkpoint intervals that need
    more memory) must be cleared in stream order before the new forward pass
    reads them: 64 pulses, 3104 states, intervals forcing reallocations."""
    s = hydrogen_like_1e(388, 7, gauge="l", seed=6)
    pulses, U, T = _batch("l", B=64, K=16, seed=4)
    X0 = np.zeros((64, s.ntot), complex)
    X0[:, 0] = 1.0
    with mpc_tdse.Context.from_system(s) as ctx:
        Js = [ctx.batch_objective(pulses, U, T, 0.0, 0.05, 300, X0, -1, ckpt_every=c)
              for c in (64, 300, 128, 257, 100, 0)]
    for J in Js[1:]:
        assert np.array_equal(J, Js[0])


def test_batch_objective_needs_forward_before_backward():
    s = hydrogen_like_1e(20, 2, seed=1)
    with mpc_tdse.Context.from_system(s) as ctx:
        with pytest.raises(mpc_tdse.MpcError):
            ctx._badj = (1, 4, 10)
            ctx.batch_objective_backward()


def test_batch_torch_autograd_function():
    import torch

    from mpc_tdse.autograd import BatchControlProblem, batch_control_objective

    s = hydrogen_like_1e(30, 3, gauge="l", seed=8)
    pulses, U, T = _batch("l", B=4, K=20, seed=2)
    X0 = np.zeros((4, s.ntot), complex)
    X0[:, 0] = 1.0
    w = np.array([1.0, -2.0, 0.5, 3.0])
    with mpc_tdse.Context.from_system(s) as ctx:
        prob = BatchControlProblem(ctx, pulses, T, 0.0, 0.1, 150, X0)
        Ut = torch.tensor(U, dtype=torch.float64, requires_grad=True)
        J = batch_control_objective(Ut, prob)
        (torch.from_numpy(w) * J).sum().backward()
        J2, G2, _ = ctx.batch_objective_gradient(pulses, U, T, 0.0, 0.1, 150, X0)
    assert np.array_equal(J.detach().numpy(), J2)
    assert np.array_equal(Ut.grad.numpy(), w[:, None] * G2)
