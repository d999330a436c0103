"""Photoelectron spectra on the GPU against a restatement of the reference's
pes program (same bins and loops) on the same full-precision coefficients,
and against the reference's own pes program (src/pes/pes.cpp compiled as it
is, tests/golden/pes.npz) including the summed -s spectra."""
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


def _ctx_for(n, eig, gauge="l"):
    """A context over the fixture's energies (the spectra need no couplings:
    zero dipole blocks)."""
    n = np.asarray(n)
    dip = np.zeros(int((n[:-1] * n[1:]).sum()))
    return mpc_tdse.Context(n, eig, dip, gauge)


def test_pes_1e_matches_the_reference_program(golden):
    """mpc_pes and mpc_pes_summed against tests/golden/pes.npz, the output
    of the reference's own src/pes/pes.cpp (6 printed digits in the 1e
    spectra, 16 in the printed numbers)."""
    f = golden("pes.npz")
    n, eig, ct = f["e1_n"], f["e1_eig"], f["e1_ct"]
    offs = np.concatenate([[0], np.cumsum(n)])
    E1 = eig[offs[1]:offs[2]]
    k = [i for i in range(n[0] - 1) if E1[i] > 0.0]
    with _ctx_for(n, eig) as ctx:
        pes, st = ctx.pes(1, ct=ct)
        grid, summed = ctx.pes_summed(1, ct=ct)
    for L in range(len(n)):
        got = np.stack([E1[k], pes[L, k]], axis=1)
        assert np.allclose(got, f[f"e1_block{L}"], rtol=5e-6, atol=0.0), L
    assert np.allclose(np.stack([grid[k], summed[k]], axis=1), f["e1_summed"], rtol=5e-6, atol=0.0)
    assert np.allclose([st["ground"], st["norm"], st["yield"]], f["e1_printed"], rtol=0.0,
                       atol=1e-12)


def test_pes_2e_matches_the_reference_program(golden):
    """2e per-block densities (16 printed digits), the -s spectrum summed over
    blocks on the L = 1 grid (6 digits) and the printed populations."""
    f = golden("pes.npz")
    n, eig, ct, thr = f["e2_n"], f["e2_eig"], f["e2_ct"], float(f["e2_threshold"])
    offs = np.concatenate([[0], np.cumsum(n)])
    with _ctx_for(n, eig, "v") as ctx:
        pes, st = ctx.pes(2, threshold=thr, ct=ct)
        grid, summed = ctx.pes_summed(2, threshold=thr, ct=ct)
    for L in range(len(n)):
        e = eig[offs[L]:offs[L + 1]]
        k = [i for i in range(1, n[L] - 1) if e[i] - thr > 0.0]
        got = np.stack([e[k] - thr, pes[L, k]], axis=1)
        assert np.allclose(got, f[f"e2_block{L}"], rtol=1e-12, atol=0.0), L
    k = [i for i in range(n[1] - 1) if grid[i] > 0.0]
    assert np.allclose(np.stack([grid[k], summed[k]], axis=1), f["e2_summed"], rtol=5e-6, atol=0.0)
    assert np.allclose([st["ground"], st["norm"], st["yield"], st["excited"]], f["e2_printed"],
                       rtol=0.0, atol=1e-12)
