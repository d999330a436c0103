"""Batched propagation (many pulses at once) against the CPU oracle.

Tolerances: batched RHS 1e-13 relative to the largest entry (the FP64
tensor-core GEMM sums in another order than the oracle's loops); adaptive
propagations: final populations within 1e-9 absolute of the oracle's
adaptive driver run with the same step control, and the same accepted-step
counts within one step.
"""
import numpy as np
import pytest

import mpc_tdse
from mpc_tdse.systems import hydrogen_like_1e, random_system

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("g", ["l", "v"])
@pytest.mark.parametrize("shape,B", [([5, 7, 6, 4, 9], 3), ([300, 513, 260, 777, 129], 37),
                                     ([298] * 6, 70), ([1, 1], 1), ([65, 64, 63], 33)])
def test_batch_rhs_matches_oracle(oracle, shape, B, g):
    s = random_system(shape, gauge=g, seed=len(shape) + B, e_max=12.0)
    rng = np.random.default_rng(B)
    X = rng.standard_normal((B, s.ntot)) + 1j * rng.standard_normal((B, s.ntot))
    F = rng.uniform(-1.5, 1.5, B)
    with mpc_tdse.Context.from_system(s) as ctx:
        got = ctx.batch_rhs(F, X)
    for b in range(B):
        want = oracle.rhs(s.n, s.eig, s.dip, g, F[b], X[b])
        scale = max(1.0, float(np.max(np.abs(want))))
        assert np.max(np.abs(got[b] - want)) <= 1e-13 * scale, (shape, B, b)


def _pulses(g, specs):
    out = []
    for Io_W, w_eV, cyc, cep in specs:
        Io, w = mpc_tdse.to_au(Io_W, w_eV)
        tau = mpc_tdse.period(w, cyc)
        out.append((mpc_tdse.pulse_setup("sine", g, Io, w, cep, cyc, tau), tau))
    return out


@pytest.mark.parametrize("path", ["auto", "streaming"])
@pytest.mark.parametrize("g", ["l", "v"])
def test_batch_adaptive_matches_oracle(oracle, g, path):
    s = hydrogen_like_1e(40, 3, gauge=g, seed=2)
    specs = [(1e14, 1.5498, 1, 0.0), (3e14, 3.0996, 2, 0.3), (5e13, 2.2, 1, 1.1),
             (2e14, 1.8, 2, 2.0), (1e13, 3.5, 1, 0.0)]
    ps = _pulses(g, specs)
    X0 = np.zeros((len(ps), s.ntot), complex)
    X0[:, 0] = 1.0
    kind = "sineEE" if g == "l" else "sineAA"
    with mpc_tdse.Context.from_system(s) as ctx:
        ctx.set_path(path)
        X, acc, rej, tf = ctx.batch_propagate([p for p, _ in ps], 0.0, [t for _, t in ps], X0,
                                              h0=0.05, dt_max=0.2, rtol=1e-10, atol=1e-10)
    for b, (p, tau) in enumerate(ps):
        xo, st = oracle.propagate_adaptive(s.n, s.eig, s.dip, g, kind, p.as_array(), 0.0, tau,
                                           0.05, 0.2, 1e-10, 1e-10, X0[b], field_mode=1)
        assert tf[b] == tau and st["t"] == tau
        assert abs(int(acc[b]) - st["accepted"]) <= 1, (b, acc[b], st)
        assert np.max(np.abs(np.abs(X[b]) ** 2 - np.abs(xo) ** 2)) < 1e-9, b
        assert abs(np.linalg.norm(X[b]) - 1.0) < 1e-13


@pytest.mark.parametrize("path", ["auto", "streaming"])
def test_batch_uneven_pulses_retire_and_compact(oracle, path):
    """70 pulses of 1..6 cycles: columns retire at different times and the
    batch is compacted repeatedly (on "auto" the last 8 pulses finish in the
    persistent resident kernel); every pulse still matches the oracle."""
    s = hydrogen_like_1e(24, 2, gauge="l", seed=4)
    rng = np.random.default_rng(5)
    specs = [(10 ** rng.uniform(13, 14.5), rng.uniform(1.0, 3.5), int(rng.integers(1, 7)),
              rng.uniform(0, 2 * np.pi)) for _ in range(70)]
    ps = _pulses("l", specs)
    X0 = np.zeros((len(ps), s.ntot), complex)
    X0[:, 0] = 1.0
    with mpc_tdse.Context.from_system(s) as ctx:
        ctx.set_path(path)
        X, acc, rej, tf = ctx.batch_propagate([p for p, _ in ps], 0.0, [t for _, t in ps], X0,
                                              h0=0.05, dt_max=0.25, rtol=1e-9, atol=1e-9)
    for b in range(0, 70, 7):
        p, tau = ps[b]
        xo, st = oracle.propagate_adaptive(s.n, s.eig, s.dip, "l", "sineEE", p.as_array(), 0.0,
                                           tau, 0.05, 0.25, 1e-9, 1e-9, X0[b], field_mode=1)
        assert tf[b] == tau
        assert abs(int(acc[b]) - st["accepted"]) <= 1
        assert np.max(np.abs(np.abs(X[b]) ** 2 - np.abs(xo) ** 2)) < 1e-8


@pytest.mark.parametrize("B", [1, 5])
def test_batch_resident_many_rows_per_cta(oracle, B):
    """A system with more than 16 rows per CTA (several register row groups
    in the resident kernel) and a velocity-gauge coupling: the persistent
    resident launch against the oracle's adaptive driver."""
    s = hydrogen_like_1e(400, 5, gauge="v", seed=7)   # 2400 states: 17 rows on some CTAs
    specs = [(1e14, 1.5498 + 0.4 * b, 1, 0.2 * b) for b in range(B)]
    ps = _pulses("v", specs)
    t_end = [6.0] * B
    X0 = np.zeros((B, s.ntot), complex)
    X0[:, 0] = 1.0
    with mpc_tdse.Context.from_system(s) as ctx:
        X, acc, rej, tf = ctx.batch_propagate([p for p, _ in ps], 0.0, t_end, X0,
                                              h0=0.02, dt_max=0.05, rtol=1e-10, atol=1e-10)
    for b, (p, tau) in enumerate(ps):
        xo, st = oracle.propagate_adaptive(s.n, s.eig, s.dip, "v", "sineAA", p.as_array(), 0.0,
                                           t_end[b], 0.02, 0.05, 1e-10, 1e-10, X0[b],
                                           field_mode=1)
        assert tf[b] == t_end[b]
        assert abs(int(acc[b]) - st["accepted"]) <= 1, (b, acc[b], st)
        assert np.max(np.abs(np.abs(X[b]) ** 2 - np.abs(xo) ** 2)) < 1e-9, b


def test_batch_resident_and_streamed_paths_agree():
    """8 pulses on the 1e hydrogen shapes through both batched paths: same
    accepted-step counts (within one) and populations within 1e-11."""
    s = hydrogen_like_1e(298, 5, gauge="l", seed=3)
    specs = [(10 ** (13 + 0.2 * b), 1.2 + 0.3 * b, 2, 0.4 * b) for b in range(8)]
    ps = _pulses("l", specs)
    t_end = [min(tau, 60.0) for _, tau in ps]
    X0 = np.zeros((8, s.ntot), complex)
    X0[:, 0] = 1.0
    out = {}
    for path in ("auto", "streaming"):
        with mpc_tdse.Context.from_system(s) as ctx:
            ctx.set_path(path)
            out[path] = ctx.batch_propagate([p for p, _ in ps], 0.0, t_end, X0, h0=0.05,
                                            dt_max=0.1, rtol=1e-10, atol=1e-10)
    Xa, acca, _, tfa = out["auto"]
    Xs, accs, _, tfs = out["streaming"]
    assert np.array_equal(tfa, tfs)
    assert np.max(np.abs(acca.astype(int) - accs.astype(int))) <= 1
    assert np.max(np.abs(np.abs(Xa) ** 2 - np.abs(Xs) ** 2)) < 1e-11


def test_autotune_table_and_variants_bit_identical(monkeypatch):
    """The autotuner reports one row per width; results do not depend on the
    tile chosen (every variant sums in the same order) nor on whether the
    attempt groups run as captured CUDA graphs."""
    s = hydrogen_like_1e(120, 4, gauge="l", seed=9)
    rng = np.random.default_rng(3)
    specs = [(10 ** rng.uniform(13, 14), rng.uniform(1.5, 3.0), 1, rng.uniform(0, 6))
             for _ in range(40)]
    ps = _pulses("l", specs)
    t_end = [min(tau, 20.0) for _, tau in ps]
    X0 = np.zeros((len(ps), s.ntot), complex)
    X0[:, 0] = 1.0

    def run(env):
        for k in ("MPC_NO_AUTOTUNE", "MPC_NO_GRAPH"):
            monkeypatch.delenv(k, raising=False)
        for k in env:
            monkeypatch.setenv(k, "1")
        with mpc_tdse.Context.from_system(s) as ctx:
            ctx.set_path("streaming")
            tab = None if env else ctx.batch_autotune(len(ps))
            return ctx.batch_propagate([p for p, _ in ps], 0.0, t_end, X0, h0=0.05, dt_max=0.2,
                                       rtol=1e-10, atol=1e-10), tab

    (Xa, acca, _, _), tab = run([])
    assert [r[0] for r in tab] == [1, 2, 4, 8, 16, 32, 64]
    assert all(r[1] in (16, 32, 64) and r[2] in (3, 6) and r[3] in (0, 1) and r[4] > 0
               for r in tab)
    for env in (["MPC_NO_AUTOTUNE"], ["MPC_NO_GRAPH"], ["MPC_NO_AUTOTUNE", "MPC_NO_GRAPH"]):
        (Xb, accb, _, _), _ = run(env)
        assert np.array_equal(acca, accb), env
        assert np.array_equal(Xa, Xb), env


def test_every_tile_variant_gives_the_same_bits(monkeypatch):
    """MPC_BATCH_VARIANT pins one of the nine stage-GEMM variants (column
    tile 16/32/64 x pipeline depth, with or without the P/Q halves in two
    CTAs): the batched forward, the batched adjoint and the fixed step's
    Horner products must not change by a bit, on a 2e system whose blocks have
    different sizes and row-tile tails."""
    from mpc_tdse.systems import helium_like_2e

    s = helium_like_2e((70, 90, 100), gauge="v", seed=4)
    rng = np.random.default_rng(8)
    specs = [(10 ** rng.uniform(13.5, 14.5), rng.uniform(1.5, 3.0), 1, rng.uniform(0, 6))
             for _ in range(11)]
    ps = _pulses("v", specs)
    pulses = [p for p, _ in ps]
    t_end = [min(tau, 8.0) for _, tau in ps]
    X0 = np.zeros((len(ps), s.ntot), complex)
    X0[:, 0] = 1.0
    U = np.stack([rng.standard_normal(24) * 0.01 * p.Eo for p in pulses])
    T = np.full(len(ps), 6.0)
    out = []
    for v in range(9):
        monkeypatch.setenv("MPC_BATCH_VARIANT", str(v))
        with mpc_tdse.Context.from_system(s) as ctx:
            ctx.set_path("streaming")
            X, acc, rej, _ = ctx.batch_propagate(pulses, 0.0, t_end, X0, h0=0.05, dt_max=0.15,
                                                 rtol=1e-10, atol=1e-10)
            J, G, Fb = ctx.batch_objective_gradient(pulses, U, T, 0.0, 0.1, 60, X0, -1,
                                                    ckpt_every=16)
            # the fixed step's Horner products, one launch each on variant v
            Xf, pf, nf = ctx.batch_advance(pulses, 0.0, 0.05, [30 + 3 * b for b in range(11)],
                                           X0, history=True)
        out.append((X, acc, rej, J, G, Fb, Xf, pf, nf))
    for v in range(1, 9):
        for a, b in zip(out[0], out[v]):
            assert np.array_equal(a, b, equal_nan=True), v


def test_single_pulse_adaptive_and_batch_names():
    """mpc_propagate_adaptive is the batched path with one pulse, and
    mpc_propagate_batch is mpc_batch_propagate: the same bits."""
    import ctypes as C

    s = hydrogen_like_1e(60, 3, gauge="l", seed=5)
    ps = _pulses("l", [(2e13, 1.8, 1, 0.4), (5e13, 2.4, 1, 1.1)])
    X0 = np.zeros((2, s.ntot), complex)
    X0[:, 0] = 1.0
    t_end = [min(tau, 15.0) for _, tau in ps]
    with mpc_tdse.Context.from_system(s) as ctx:
        ctx.set_path("streaming")
        Xb, accb, rejb, tfb = ctx.batch_propagate([ps[0][0]], 0.0, [t_end[0]], X0[:1], h0=0.05,
                                                  dt_max=0.2)
        x1, acc1, rej1, tf1 = ctx.propagate_adaptive(ps[0][0], 0.0, t_end[0], X0[0], h0=0.05,
                                                     dt_max=0.2)
        assert np.array_equal(Xb[0], x1) and accb[0] == acc1 and rejb[0] == rej1
        assert tfb[0] == tf1
        L = mpc_tdse.lib()
        arr = (mpc_tdse.Pulse * 2)(*[p for p, _ in ps])
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int)
        t0 = np.zeros(2)
        te = np.array(t_end)
        res = []
        for fn in (L.mpc_batch_propagate, L.mpc_propagate_batch):
            xf = X0.view(np.float64).copy()
            acc = np.zeros(2, np.int32)
            rej = np.zeros(2, np.int32)
            tf = np.zeros(2)
            rc = fn(ctx._h, 2, arr, t0.ctypes.data_as(dp), te.ctypes.data_as(dp), 0.05, 0.2,
                    1e-10, 1e-10, 0, xf.ctypes.data_as(dp), acc.ctypes.data_as(ip),
                    rej.ctypes.data_as(ip), tf.ctypes.data_as(dp))
            assert rc == 0, mpc_tdse.last_error()
            res.append((xf, acc, rej, tf))
        for a, b in zip(*res):
            assert np.array_equal(a, b)
