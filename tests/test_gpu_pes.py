"""Photoelectron spectra on the GPU against a restatement of the reference's
pes program (same bins and loops) on the same full-precision coefficients."""
import numpy as np
import pytest

import mpc_tdse
from mpc_tdse.structure1e import hydrogen
from mpc_tdse.systems import helium_like_2e
from oracle import pes_reference

pytestmark = pytest.mark.gpu


def test_pes_1e_matches_reference_restatement():
    s = hydrogen(n=80, k=9, R=60.0, l_max=3, gauge="l", states=[70] * 4)
    x0 = np.zeros(s.ntot, complex)
    x0[0] = 1.0
    Io, w = mpc_tdse.to_au(3e14, 3.0)
    p = mpc_tdse.pulse_setup("sine", "l", Io, w, 0.0, 3, mpc_tdse.period(w, 3))
    with mpc_tdse.Context.from_system(s) as ctx:
        ct, *_ = ctx.propagate(p, 0.0, 0.05, 600, x0)
        pes, st = ctx.pes(1)
        pes2, st2 = ctx.pes(1, ct=ct)
    ref, g, nrm, y, _ = pes_reference(s.n, s.eig, ct, 1)
    assert np.max(np.abs(pes - ref)) <= 1e-12 * max(1.0, np.max(np.abs(ref)))
    assert abs(st["ground"] - g) < 1e-15 and abs(st["norm"] - nrm) < 1e-13
    assert abs(st["yield"] - y) < 1e-13 and st["yield"] > 0
    assert np.array_equal(pes, pes2)


def test_pes_2e_matches_reference_restatement():
    s = helium_like_2e((50, 60, 55), gauge="v", seed=2)
    rng = np.random.default_rng(0)
    ct = rng.standard_normal(s.ntot) + 1j * rng.standard_normal(s.ntot)
    ct /= np.linalg.norm(ct)
    with mpc_tdse.Context.from_system(s) as ctx:
        pes, st = ctx.pes(2, threshold=-2.0, ct=ct)
    ref, g, nrm, y, exc = pes_reference(s.n, s.eig, ct, 2, threshold=-2.0)
    assert np.max(np.abs(pes - ref)) <= 1e-12 * max(1.0, np.max(np.abs(ref)))
    assert abs(st["yield"] - y) < 1e-13 and abs(st["excited"] - exc) < 1e-13
