"""Known answers for the GPU propagation that need no reference run: a
two-level (Rabi) system against the exact exponential of its 2x2 generator,
field-free evolution against the exact phases exp(-i e t), and the norm before
each renormalisation (an RKF78 step is not exactly unitary; its drift is the
truncation error).

Tolerances: 1e-12 absolute on the coefficients (dt = 0.01..0.02 keeps the
RKF78 truncation far below rounding), 1e-10 on |norm - 1| per step at
dt = 0.1 inside the stability interval.
"""
import numpy as np
import pytest
from scipy.linalg import expm

import mpc_tdse
from mpc_tdse.systems import random_system

pytestmark = pytest.mark.gpu


def _generator(gauge, w0, d, F):
    """dc/dt = M c for two states (block L=0: energy 0, L=1: energy w0,
    dipole block [[d]]): length gauge M = -i [[0, F d], [F d, w0]];
    velocity gauge M = [[0, -F d], [F d, -i w0]] (D_0 couples with a minus
    sign into block 0 and a plus sign into block 1)."""
    if gauge == "l":
        return -1j * np.array([[0.0, F * d], [F * d, w0]])
    return np.array([[0.0, -F * d], [F * d, -1j * w0]])


@pytest.mark.parametrize("gauge", ["l", "v"])
def test_rabi_two_level_matches_exact_exponential(gauge):
    """Constant field through mpc_rk78_step (one fixed step at a frozen F)."""
    w0, d, F, dt, steps = 0.35, 1.3, 0.2, 0.02, 400
    with mpc_tdse.Context([1, 1], [0.0, w0], [d], gauge) as ctx:
        x = np.array([1.0 + 0j, 0.0 + 0j])
        for _ in range(steps):
            x = ctx.rk78_step(F, dt, x)
    want = expm(_generator(gauge, w0, d, F) * dt * steps) @ np.array([1.0, 0.0])
    assert np.max(np.abs(x - want)) < 1e-12
    # a Rabi oscillation really happened
    assert abs(x[1]) > 0.3


@pytest.mark.parametrize("gauge", ["l", "v"])
@pytest.mark.parametrize("path", ["streaming", "resident"])
def test_field_free_phases_are_exact(gauge, path):
    """A zero-amplitude pulse through the full propagation loop (both paths):
    every coefficient only turns by exp(-i e t)."""
    s = random_system([40, 57, 33], gauge=gauge, seed=11, e_max=4.0)
    rng = np.random.default_rng(12)
    x0 = rng.standard_normal(s.ntot) + 1j * rng.standard_normal(s.ntot)
    x0 /= np.linalg.norm(x0)
    dt, steps = 0.01, 300
    _, w = mpc_tdse.to_au(1e14, 1.5498)
    p = mpc_tdse.pulse_setup("sine", gauge, 0.0, w, 0.0, 2, mpc_tdse.period(w, 2))
    with mpc_tdse.Context.from_system(s) as ctx:
        ctx.set_path(path)
        x, _, fld, _ = ctx.propagate(p, 0.0, dt, steps, x0)
    assert np.all(fld == 0.0)
    want = np.exp(-1j * s.eig * dt * steps) * x0
    assert np.max(np.abs(x - want)) < 1e-12


@pytest.mark.parametrize("path", ["streaming", "resident"])
def test_norm_drift_before_renormalisation(path):
    from mpc_tdse.systems import hydrogen_like_1e

    s = hydrogen_like_1e(60, 3, gauge="l", seed=2)
    Io, w = mpc_tdse.to_au(1e14, 1.5498)
    p = mpc_tdse.pulse_setup("sine", "l", Io, w, 0.0, 2, mpc_tdse.period(w, 2))
    x0 = np.zeros(s.ntot, complex)
    x0[0] = 1.0
    with mpc_tdse.Context.from_system(s) as ctx:
        ctx.set_path(path)
        ct, pop, fld, nrm = ctx.propagate(p, 0.0, 0.1, 600, x0)
    assert np.max(np.abs(nrm - 1.0)) < 1e-10
    assert abs(np.linalg.norm(ct) - 1.0) < 1e-14
