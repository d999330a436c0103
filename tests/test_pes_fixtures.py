"""The PES restatement against the reference's own pes program.

tests/golden/pes.npz holds what the reference's src/pes/pes.cpp
(pes::genPES1e / genPES2e with -s) writes and prints for seeded coefficients
(made by tests/golden/make_golden.py from oracle/_ref/libref_pes.so).  The
reference writes the 1e spectra and the 2e summed spectrum with the stream's
default 6 significant digits, the 2e per-block spectra and every printed
number with 16: the tolerances follow (5e-6 relative: half a unit of the sixth digit; 1e-12).
"""
import numpy as np

from oracle import pes_reference, pes_summed_reference


def _rows_1e(E1, values, n0):
    k = [i for i in range(n0 - 1) if E1[i] > 0.0]
    return np.stack([E1[k], values[k]], axis=1)


def test_1e_spectra_match_the_reference_program(golden):
    f = golden("pes.npz")
    n, eig, ct = f["e1_n"], f["e1_eig"], f["e1_ct"]
    pes, g, nrm, y, _ = pes_reference(n, eig, ct, 1)
    offs = np.concatenate([[0], np.cumsum(n)])
    E1 = eig[offs[1]:offs[2]]
    for L in range(len(n)):
        want = f[f"e1_block{L}"]
        got = _rows_1e(E1, pes[L], n[0])
        assert got.shape == want.shape
        assert np.allclose(got, want, rtol=5e-6, atol=0.0), L
    grid, summed = pes_summed_reference(n, eig, ct, 1)
    assert np.allclose(_rows_1e(grid, summed, n[0]), f["e1_summed"], rtol=5e-6, atol=0.0)
    assert np.allclose([g, nrm, y], f["e1_printed"], rtol=0.0, atol=1e-12)


def test_2e_spectra_match_the_reference_program(golden):
    f = golden("pes.npz")
    n, eig, ct, thr = f["e2_n"], f["e2_eig"], f["e2_ct"], float(f["e2_threshold"])
    pes, g, nrm, y, exc = pes_reference(n, eig, ct, 2, threshold=thr)
    offs = np.concatenate([[0], np.cumsum(n)])
    for L in range(len(n)):
        e = eig[offs[L]:offs[L + 1]]
        k = [i for i in range(1, n[L] - 1) if e[i] - thr > 0.0]
        got = np.stack([e[k] - thr, pes[L, k]], axis=1)
        assert np.allclose(got, f[f"e2_block{L}"], rtol=1e-12, atol=0.0), L
    grid, summed = pes_summed_reference(n, eig, ct, 2, threshold=thr)
    k = [i for i in range(n[1] - 1) if grid[i] > 0.0]
    assert np.allclose(np.stack([grid[k], summed[k]], axis=1), f["e2_summed"], rtol=5e-6, atol=0.0)
    assert np.allclose([g, nrm, y, exc], f["e2_printed"], rtol=0.0, atol=1e-12)
