"""GPU parity: libmpc_tdse.so (through its C ABI) against the CPU oracle and
against golden outputs of the reference's own code.

Tolerances (absolute, on populations |c|^2 and coefficients c):
  single RHS / single step: 1e-13 relative to the largest entry;
  short propagations vs oracle: 1e-11;
  full reference-semantics pulses vs the reference (golden): 1e-9, the bar
  the propagation must meet.
"""
import numpy as np
import pytest

import mpc_tdse
from mpc_tdse.systems import helium_like_2e, hydrogen_like_1e, random_system

pytestmark = pytest.mark.gpu

SHAPES = {
    "tiny": [1, 1],
    "ragged": [5, 7, 6, 4, 9],
    "multistrip": [300, 513, 260, 777, 129],
    "wide": [17, 1030, 33],
    "manyblocks": [20] * 13,
    "h1e": [298] * 6,
}


def _sys(shape, g, seed=0):
    return random_system(SHAPES[shape], gauge=g, seed=seed, e_max=12.0)


def _x(n, seed=1):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    return x / np.linalg.norm(x)


@pytest.mark.parametrize("g", ["l", "v"])
@pytest.mark.parametrize("shape", list(SHAPES))
def test_rhs_matches_oracle(oracle, shape, g):
    s = _sys(shape, g)
    x = _x(s.ntot)
    with mpc_tdse.Context.from_system(s) as ctx:
        for F in (0.0, 0.053, -1.7):
            got = ctx.rhs(F, x)
            want = oracle.rhs(s.n, s.eig, s.dip, g, F, x)
            scale = max(1.0, float(np.max(np.abs(want))))
            assert np.max(np.abs(got - want)) <= 1e-13 * scale, (shape, g, F)


@pytest.mark.parametrize("g", ["l", "v"])
def test_rhs_matches_reference_golden(golden, g):
    z = golden("rhs.npz")
    n, eig, dip, x = z[f"rhs_{g}_n"], z[f"rhs_{g}_eig"], z[f"rhs_{g}_dip"], z[f"rhs_{g}_x"]
    with mpc_tdse.Context(n, eig, dip, g) as ctx:
        for F in (0.0, 0.37, -1.25):
            want = z[f"rhs_{g}_{F}"]
            got = ctx.rhs(F, x)
            assert np.max(np.abs(got - want)) <= 1e-13 * max(1.0, np.max(np.abs(want)))


@pytest.mark.parametrize("g", ["l", "v"])
@pytest.mark.parametrize("shape", ["ragged", "multistrip", "h1e"])
def test_rk78_step_matches_oracle(oracle, shape, g):
    s = _sys(shape, g, seed=5)
    x = _x(s.ntot, seed=6)
    with mpc_tdse.Context.from_system(s) as ctx:
        got = ctx.rk78_step(0.21, 0.1, x)
    want = oracle.rk78_step(s.n, s.eig, s.dip, g, 0.21, 0.1, x)
    assert np.max(np.abs(got - want)) <= 1e-13


@pytest.mark.parametrize("path", ["streaming", "resident"])
@pytest.mark.parametrize("g", ["l", "v"])
@pytest.mark.parametrize("shape", ["tiny", "ragged", "multistrip", "manyblocks", "h1e"])
def test_propagate_matches_oracle(oracle, shape, g, path):
    s = _sys(shape, g, seed=9)
    x0 = np.zeros(s.ntot, complex)
    x0[0] = 1.0
    Io, w = mpc_tdse.to_au(3e14, 1.5498)
    tau = mpc_tdse.period(w, 3)
    p = mpc_tdse.pulse_setup("sine", g, Io, w, 0.0, 3, tau)
    steps = 60
    pop_index = min(3, s.ntot - 1)
    with mpc_tdse.Context.from_system(s) as ctx:
        ctx.set_path(path)
        assert ctx.path == path
        ct, pop, fld, nrm = ctx.propagate(p, 0.0, 0.1, steps, x0, pop_index=pop_index)
    kind = "sineEE" if g == "l" else "sineAA"
    cto, popo, fldo, nrmo = oracle.propagate(s.n, s.eig, s.dip, g, kind, p.as_array(), 0.0, 0.1,
                                             steps, x0, pop_index=pop_index)
    np.testing.assert_array_equal(fld, fldo)
    assert np.max(np.abs(ct - cto)) < 1e-11
    assert np.max(np.abs(pop - popo)) < 1e-11
    assert np.max(np.abs(nrm - nrmo)) < 1e-12


@pytest.mark.parametrize("path", ["streaming", "resident"])
@pytest.mark.parametrize("case", [("l", "sine"), ("v", "sine"), ("l", "gaussian")])
def test_full_pulse_matches_reference_golden(golden, case, path):
    """A whole 2-cycle pulse (2206 steps) against the reference's propL/propV."""
    g, shape = case
    z = golden("propagate.npz")
    key = f"prop_{g}_{shape}"
    n, eig, dip = z[key + "_n"], z[key + "_eig"], z[key + "_dip"]
    steps = int(z[key + "_steps"])
    Io, w = mpc_tdse.to_au(1e14, 1.5498)
    tau = mpc_tdse.period(w, 2)
    p = mpc_tdse.pulse_setup(shape, g, Io, w, 0.0, 2, tau)
    x0 = np.zeros(int(np.sum(n)), complex)
    x0[0] = 1.0
    with mpc_tdse.Context(n, eig, dip, g) as ctx:
        ctx.set_path(path)
        ct, pop, fld, nrm = ctx.propagate(p, 0.0, 0.1, steps, x0)
    ref_ct = z[key + "_ct"]
    assert np.max(np.abs(np.abs(ct) ** 2 - np.abs(ref_ct) ** 2)) < 1e-9
    assert np.max(np.abs(z[key + "_pop"][:, 1] - pop)) < 1e-9
    np.testing.assert_allclose(z[key + "_field"][:, 1], fld, rtol=1e-5, atol=1e-12)


@pytest.mark.parametrize("path", ["streaming", "resident"])
def test_repeat_runs_are_bit_identical(path):
    s = _sys("multistrip", "v", seed=2)
    x0 = _x(s.ntot, seed=3)
    Io, w = mpc_tdse.to_au(1e14, 3.179)
    p = mpc_tdse.pulse_setup("sine", "v", Io, w, 0.0, 8, 0.0)
    with mpc_tdse.Context.from_system(s) as ctx:
        ctx.set_path(path)
        a = ctx.propagate(p, 0.0, 0.1, 25, x0)
        b = ctx.propagate(p, 0.0, 0.1, 25, x0)
    for u, v in zip(a, b):
        assert np.array_equal(u, v)


def test_unstable_dt_is_rejected():
    s = _sys("ragged", "l")
    x0 = _x(s.ntot)
    p = mpc_tdse.pulse_setup("sine", "l", 1e-3, 0.05, 0.0, 2, 0.0)
    with mpc_tdse.Context.from_system(s) as ctx:
        with pytest.raises(mpc_tdse.MpcError) as e:
            ctx.propagate(p, 0.0, 1.0, 10, x0)
    assert e.value.code == -5


def test_resident_path_is_not_taken_when_the_system_does_not_fit(he2e):
    with mpc_tdse.Context.from_system(he2e) as ctx:
        assert ctx.path == "streaming"
        with pytest.raises(mpc_tdse.MpcError):
            ctx.set_path("resident")


def test_device_resident_advance_equals_propagate():
    s = _sys("multistrip", "l", seed=4)
    x0 = np.zeros(s.ntot, complex)
    x0[0] = 1
    Io, w = mpc_tdse.to_au(2e14, 1.5498)
    p = mpc_tdse.pulse_setup("sine", "l", Io, w, 0.0, 4, 0.0)
    with mpc_tdse.Context.from_system(s) as ctx:
        ct, pop, fld, nrm = ctx.propagate(p, 0.0, 0.1, 30, x0, pop_index=2)
        ctx.state_set(x0)
        ctx.advance(p, 0.0, 0.1, 30, pop_index=2)
        ct2 = ctx.state_get()
        pop2, fld2, nrm2 = ctx.history(30)
    assert np.array_equal(ct, ct2) and np.array_equal(pop, pop2) and np.array_equal(nrm, nrm2)


@pytest.fixture(scope="module")
def he2e():
    """The 2e helium-like system at full size (L = 0..3, 18000 states,
    61.8M dipole elements, 495 MB)."""
    return helium_like_2e(gauge="v", seed=0)


def test_full_size_2e_rhs_matches_oracle(oracle, he2e):
    s = he2e
    x = _x(s.ntot, seed=11)
    oracle.use_openblas()
    try:
        want = oracle.rhs(s.n, s.eig, s.dip, "v", 1.02, x)
    finally:
        oracle.use_plain_loops()
    with mpc_tdse.Context.from_system(s) as ctx:
        got = ctx.rhs(1.02, x)
    assert np.max(np.abs(got - want)) <= 1e-12 * max(1.0, np.max(np.abs(want)))


def test_full_size_2e_field_free_is_stability_polynomial(oracle, he2e):
    """Size-independent property at full size: with F = 0 every coefficient
    is multiplied by R(-i e dt) each step, then the state is renormalised."""
    s = he2e
    A, b8, _, _ = oracle.tableau()
    x0 = _x(s.ntot, seed=12)
    dt, steps = 0.1, 40
    z = -1j * s.eig * dt
    R = np.ones_like(z)
    for k in range(13):
        R = R + z ** (k + 1) * (b8 @ np.linalg.matrix_power(A, k) @ np.ones(13))
    x = x0.copy()
    for _ in range(steps):
        x = R * x
        x /= np.linalg.norm(x)
    p = mpc_tdse.pulse_setup("sine", "v", 0.0, 0.1168, 0.0, 8, 0.0)  # Io = 0: F(t) = 0
    with mpc_tdse.Context.from_system(s) as ctx:
        ct, pop, fld, nrm = ctx.propagate(p, 0.0, dt, steps, x0)
    assert np.all(fld == 0.0)
    assert np.max(np.abs(ct - x)) < 1e-12


def test_full_size_2e_short_propagation_matches_oracle(oracle, he2e):
    s = he2e
    x0 = np.zeros(s.ntot, complex)
    x0[0] = 1.0
    Io, w = mpc_tdse.to_au(5e14, 3.179)
    tau = mpc_tdse.period(w, 8)
    p = mpc_tdse.pulse_setup("sine", "v", Io, w, 0.0, 8, tau)
    t0, steps = 200.0, 3  # mid-pulse, strong field
    with mpc_tdse.Context.from_system(s) as ctx:
        ct, pop, fld, nrm = ctx.propagate(p, t0, 0.1, steps, x0)
    oracle.use_openblas()
    try:
        cto, popo, fldo, nrmo = oracle.propagate(s.n, s.eig, s.dip, "v", "sineAA", p.as_array(),
                                                 t0, 0.1, steps, x0)
    finally:
        oracle.use_plain_loops()
    assert np.max(np.abs(np.abs(ct) ** 2 - np.abs(cto) ** 2)) < 1e-12
    assert np.max(np.abs(nrm - nrmo)) < 1e-12


@pytest.mark.parametrize("gauge", ["l", "v"])
def test_horner_steps_equal_stage_form(monkeypatch, gauge):
    """The streamed path's fixed step as the 12 Horner products of the RKF78
    stability polynomial against the same step as 13 stages (MPC_STAGE_FORM):
    the same frozen-field step, so the same state up to rounding, over a
    whole short pulse; both against the oracle."""
    s = _sys("multistrip", gauge, seed=7)
    x0 = _x(s.ntot, seed=8)
    Io, w = mpc_tdse.to_au(2e14, 1.5498)
    p = mpc_tdse.pulse_setup("sine", gauge, Io, w, 0.0, 2, 0.0)
    out = []
    for stage_form in (False, True):
        if stage_form:
            monkeypatch.setenv("MPC_STAGE_FORM", "1")
        with mpc_tdse.Context.from_system(s) as ctx:
            ctx.set_path("streaming")
            out.append(ctx.propagate(p, 0.0, 0.1, 120, x0))
    (ct_h, pop_h, fld_h, nrm_h), (ct_s, pop_s, fld_s, nrm_s) = out
    assert np.array_equal(fld_h, fld_s)
    assert np.max(np.abs(ct_h - ct_s)) < 1e-12
    assert np.max(np.abs(pop_h - pop_s)) < 1e-12
    assert np.max(np.abs(nrm_h - nrm_s)) < 1e-12
    assert not np.array_equal(ct_h, ct_s)   # the two forms did run


def test_l2_keep_hint_changes_no_bit(monkeypatch):
    """The dipole stream's L2 evict-last share (MPC_L2_KEEP_MB) is a cache
    hint only: the same bits with none of the couplings kept and with all."""
    s = _sys("multistrip", "l", seed=9)
    x0 = _x(s.ntot, seed=10)
    Io, w = mpc_tdse.to_au(1e14, 1.5498)
    p = mpc_tdse.pulse_setup("sine", "l", Io, w, 0.0, 2, 0.0)
    out = []
    for keep in ("0", "100000"):
        monkeypatch.setenv("MPC_L2_KEEP_MB", keep)
        with mpc_tdse.Context.from_system(s) as ctx:
            ctx.set_path("streaming")
            out.append(ctx.propagate(p, 0.0, 0.1, 40, x0))
    for u, v in zip(*out):
        assert np.array_equal(u, v)
