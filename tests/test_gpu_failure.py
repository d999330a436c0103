"""Failure detection on the GPU, in forms that neither fault nor hang it.

* Bounded waits: the persistent kernels' grid barriers take their wait limit
  from the context (mpc_ctx_set_wait_limit).  A test sets 1 ms and injects a
  barrier that no CTA can complete (mpc_ctx_inject_barrier_timeout: the
  targets sit one arrival beyond the grid), so every CTA's first wait runs
  out, the kernel returns, and the call reports MPC_ERR_DEVICE with the
  wait-timeout status.  The same context then propagates normally and
  matches the CPU oracle: the status word was cleared and nothing was lost.
* Non-finite data: a NaN planted in the host coefficient vector before the
  upload makes the norm reduction raise the non-finite status; the call
  returns MPC_ERR_DEVICE and the next call on clean data succeeds.
"""
import numpy as np
import pytest

import mpc_tdse
from mpc_tdse.systems import hydrogen_like_1e, random_system

pytestmark = pytest.mark.gpu


def _pulse(gauge="l", cycles=2):
    Io, w = mpc_tdse.to_au(1e14, 1.5498)
    return mpc_tdse.pulse_setup("sine", gauge, Io, w, 0.0, cycles, mpc_tdse.period(w, cycles))


def test_resident_barrier_timeout_is_reported_and_context_recovers(oracle):
    s = random_system([60, 70, 50], gauge="l", seed=3, e_max=8.0)
    p = _pulse()
    x0 = np.zeros(s.ntot, complex)
    x0[0] = 1.0
    with mpc_tdse.Context.from_system(s) as ctx:
        ctx.set_path("resident")
        ctx.set_wait_limit(1e-3)
        ctx.inject_barrier_timeout()
        with pytest.raises(mpc_tdse.MpcError) as ei:
            ctx.propagate(p, 0.0, 0.1, 30, x0)
        assert ei.value.code == -3
        assert "wait timeout" in str(ei.value)
        # the hook was one-shot; the same context is usable again
        ctx.set_wait_limit(2.0)
        ct, pop, fld, _ = ctx.propagate(p, 0.0, 0.1, 30, x0)
    ct_o, pop_o, fld_o, _ = oracle.propagate(s.n, s.eig, s.dip, "l", "sineEE", p.as_array(), 0.0,
                                             0.1, 30, x0)
    assert np.array_equal(fld, fld_o)
    assert np.max(np.abs(np.abs(ct) ** 2 - np.abs(ct_o) ** 2)) < 1e-9


def test_adjoint_forward_barrier_timeout_is_reported():
    s = random_system([60, 70, 50], gauge="l", seed=4, e_max=8.0)
    p = _pulse()
    x0 = np.zeros(s.ntot, complex)
    x0[0] = 1.0
    u = np.linspace(-1, 1, 8) * 1e-3
    T = mpc_tdse.period(p.w, 2)
    with mpc_tdse.Context.from_system(s) as ctx:
        ctx.set_path("resident")
        J0, g0, _ = ctx.objective_gradient(p, u, T, 0.0, 0.1, 40, x0, -1, 16)
        ctx.set_wait_limit(1e-3)
        ctx.inject_barrier_timeout()
        with pytest.raises(mpc_tdse.MpcError) as ei:
            ctx.objective(p, u, T, 0.0, 0.1, 40, x0, -1, 16)
        assert ei.value.code == -3
        ctx.set_wait_limit(2.0)
        # the reverse pass's persistent launch
        ctx.objective(p, u, T, 0.0, 0.1, 40, x0, -1, 16)
        ctx.set_wait_limit(1e-3)
        ctx.inject_barrier_timeout()
        with pytest.raises(mpc_tdse.MpcError) as ei:
            ctx.objective_backward()
        assert ei.value.code == -3
        ctx.set_wait_limit(2.0)
        J1, g1, _ = ctx.objective_gradient(p, u, T, 0.0, 0.1, 40, x0, -1, 16)
    assert J1 == J0
    assert np.array_equal(g1, g0)


def test_batched_resident_tail_barrier_timeout_is_reported():
    # 3 blocks of 80 states: every one of the 148 CTAs of the resident batched
    # kernel gets rows (a much smaller system does not take that path)
    h = hydrogen_like_1e(80, 2, gauge="l", seed=4)
    x = np.zeros(h.ntot, complex)
    x[0] = 1.0
    T = 5.0
    ps = [_pulse(cycles=1), _pulse(cycles=1)]
    with mpc_tdse.Context.from_system(h) as ctx:
        X0, acc0, _, _ = ctx.batch_propagate(ps, 0.0, [T, T], np.stack([x, x]), h0=0.05,
                                             dt_max=0.2)
        ctx.set_wait_limit(1e-3)
        ctx.inject_barrier_timeout()
        with pytest.raises(mpc_tdse.MpcError) as ei:
            ctx.batch_propagate(ps, 0.0, [T, T], np.stack([x, x]), h0=0.05, dt_max=0.2)
        assert ei.value.code == -3
        assert "0x1" in str(ei.value)
        ctx.set_wait_limit(2.0)
        X1, acc1, _, _ = ctx.batch_propagate(ps, 0.0, [T, T], np.stack([x, x]), h0=0.05,
                                             dt_max=0.2)
    assert np.array_equal(acc0, acc1)
    assert np.array_equal(X0, X1)


def test_persistent_batched_step_dependency_timeout_is_reported(monkeypatch):
    """The batched fixed step's persistent launch (Horner products flowing
    from one to the next on per-column progress counters): an injected
    dependency that cannot complete runs out after the limit, the other CTAs
    stop on the raised status, the call reports it, and the context recovers."""
    from mpc_tdse.structure1e import hydrogen

    # 1752 states (30 row tiles): 96 pulses give enough tiles per product for
    # the persistent launch
    s = hydrogen(n=300, k=9, R=200.0, l_max=5, gauge="l", states=[292] * 6)
    Io, w = mpc_tdse.to_au(1e14, 1.5498)
    tau = mpc_tdse.period(w, 1)
    ps = [mpc_tdse.pulse_setup("sine", "l", Io * (1 + 0.01 * b), w, 0.0, 1, tau)
          for b in range(96)]
    X0 = np.zeros((96, s.ntot), complex)
    X0[:, 0] = 1.0
    steps = [30 + (b % 7) for b in range(96)]
    # the persistent launch at every width
    monkeypatch.setenv("MPC_FORCE_PERSIST", "1")
    with mpc_tdse.Context.from_system(s) as ctx:
        ctx.set_path("streaming")   # every step on the GEMM path
        Xa = ctx.batch_advance(ps, 0.0, 0.05, steps, X0)
        ctx.set_wait_limit(1e-3)
        ctx.inject_barrier_timeout()
        with pytest.raises(mpc_tdse.MpcError) as ei:
            ctx.batch_advance(ps, 0.0, 0.05, steps, X0)
        assert ei.value.code == -3
        ctx.set_wait_limit(2.0)
        Xb = ctx.batch_advance(ps, 0.0, 0.05, steps, X0)
    assert np.array_equal(Xa, Xb)


@pytest.mark.parametrize("path", ["streaming", "resident"])
def test_nan_in_host_state_raises_nonfinite_status(path):
    s = random_system([40, 57, 33], gauge="v", seed=11, e_max=4.0)
    p = _pulse("v")
    x0 = np.zeros(s.ntot, complex)
    x0[0] = 1.0
    bad = x0.copy()
    bad[17] = np.nan
    with mpc_tdse.Context.from_system(s) as ctx:
        ctx.set_path(path)
        with pytest.raises(mpc_tdse.MpcError) as ei:
            ctx.propagate(p, 0.0, 0.1, 12, bad)
        assert ei.value.code == -3
        assert "non-finite" in str(ei.value)
        ct, _, _, nrm = ctx.propagate(p, 0.0, 0.1, 12, x0)
    assert np.all(np.isfinite(ct))
    assert np.max(np.abs(nrm - 1.0)) < 1e-10
