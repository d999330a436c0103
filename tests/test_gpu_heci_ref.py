"""Parity at the headline benchmark's own size, against the reference's own
propagation loop.

The system is genuine He CI from the restated 2e structure chain (400
B-splines of order 9, R = 150, l <= 4, inner electron n <= 3, total L = 0..3;
the CI states below 20 a.u.: 19,053 states, 547 MB of FP64 couplings), velocity
gauge, with the 8-cycle 390 nm 5e14 W/cm^2 sin^2 pulse at dt = 0.1.  From the
library's own state in the middle of the pulse, where the field is strongest,
60 steps run through the reference's `tdse::propV` (src/tdse/tdse.cpp:186-215,
built from its own source into oracle/_ref, OpenBLAS on the host cores) and
through the library's streamed path, both as the 12 Horner products it uses by
default and as the 13 stages (MPC_STAGE_FORM), all three from the same state:
coefficients within 1e-12 of the reference, populations and the
pre-renormalisation norms of the two forms within 1e-12 of each other.
"""
import os
import tempfile

import numpy as np
import pytest

import mpc_tdse
from oracle import Reference

pytestmark = pytest.mark.gpu

W_EV, IO, CYCLES, DT, NSTEPS = 3.179, 5e14, 8, 0.1, 60


@pytest.fixture(scope="module")
def heci():
    from mpc_tdse import structure2e

    s, _ = structure2e.helium(n=400, R=150.0, Z=2.0, l_max=4, L_max=3, n_inner=3,
                              n_outer=360, gauge="v", device="cuda", e_cut=20.0)
    assert s.ntot > 18000
    return s


def test_heci_mid_pulse_steps_match_reference(heci, monkeypatch):
    if not Reference.available():
        pytest.skip("reference build not present")
    s = heci
    Iau, wau = mpc_tdse.to_au(IO, W_EV)
    tau = mpc_tdse.period(wau, CYCLES)
    p = mpc_tdse.pulse_setup("sine", "v", Iau, wau, 0.0, CYCLES, tau)
    ref = Reference()
    ref.use_openblas(os.cpu_count() or 1)
    total = ref.steps(W_EV, CYCLES, 0.0, DT)
    k_mid = total // 2 - NSTEPS // 2
    x0 = np.zeros(s.ntot, complex)
    x0[0] = 1.0
    with mpc_tdse.Context.from_system(s) as ctx:
        assert ctx.path == "streaming"
        x_mid = ctx.propagate(p, 0.0, DT, k_mid, x0, history=False)
        ct_h, pop_h, _, nrm_h = ctx.propagate(p, k_mid * DT, DT, NSTEPS, x_mid)
    monkeypatch.setenv("MPC_STAGE_FORM", "1")
    with mpc_tdse.Context.from_system(s) as ctx:
        x_mid_s = ctx.propagate(p, 0.0, DT, k_mid, x0, history=False)
        ct_s, pop_s, _, nrm_s = ctx.propagate(p, k_mid * DT, DT, NSTEPS, x_mid)
    # (over the first half of the pulse, 2,000+ steps at dt * max|E| = 2.0, the
    # two forms' rounding differences grow to 4e-9..2e-8 in the coefficients; the
    # comparison below starts both from the same mid-pulse state)
    drift = float(np.max(np.abs(x_mid - x_mid_s)))
    with tempfile.TemporaryDirectory() as d:
        ct_r = ref.propagate(s.n, s.eig, s.dip, "v", "sine", IO, W_EV, CYCLES, k_mid * DT, DT,
                             NSTEPS, x_mid, os.path.join(d, "he"))
    err_h = float(np.max(np.abs(ct_h - ct_r)))
    err_s = float(np.max(np.abs(ct_s - ct_r)))
    print(f"\nHe CI {s.ntot} states, steps {k_mid}..{k_mid + NSTEPS} of {total}: "
          f"max |c - reference| = {err_h:.2e} (Horner products), {err_s:.2e} (stages); "
          f"the two forms after the first {k_mid} steps: {drift:.2e}")
    assert err_h < 1e-12 and err_s < 1e-12
    assert np.max(np.abs(np.abs(ct_h) ** 2 - np.abs(ct_r) ** 2)) < 1e-12
    assert np.max(np.abs(pop_h - pop_s)) < 1e-12
    assert np.max(np.abs(nrm_h - nrm_s)) < 1e-12
