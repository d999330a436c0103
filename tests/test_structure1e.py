"""The 1e structure restatement (h1e/w1e/d1e) against hydrogen's analytic
answers: bound energies -Z^2/(2 n^2), the 1s-2p length-gauge dipole
(128 sqrt(6)/243 times the angular factor 1/sqrt(3)), and the
velocity/length relation <a|p|b> = (E_b - E_a) <a|r|b> for exact eigenstates."""
import numpy as np

from mpc_tdse import io
from mpc_tdse.structure1e import dipoles_1e, hydrogen, solve_1e, write_1e_files


def test_hydrogen_spectrum_and_dipoles():
    t, Es, Cs = solve_1e(n=60, k=9, R=40.0, Z=1.0, l_max=2)
    # 1s, 2s, 2p are converged in a 40 a.u. box; 3d to 1e-6 (higher states
    # feel the box wall)
    assert abs(Es[0][0] + 0.5) < 1e-9 and abs(Es[0][1] + 0.125) < 1e-9
    assert abs(Es[1][0] + 0.125) < 1e-9
    assert abs(Es[2][0] + 0.5 / 9) < 1e-6
    Dl = dipoles_1e(t, 9, Cs, 40.0, "l")
    Dv = dipoles_1e(t, 9, Cs, 40.0, "v")
    assert abs(Dl[0][0, 0] - 128 * np.sqrt(6) / 243 / np.sqrt(3)) < 1e-9
    assert abs(Dv[0][0, 0] / Dl[0][0, 0] - (Es[1][0] - Es[0][0])) < 1e-9
    # positive slope at the origin for every state
    assert np.all(Cs[0][:, 1] > 0)


def test_truncated_system_and_files(tmp_path):
    s = hydrogen(n=40, k=7, R=30.0, l_max=2, gauge="v", states=[30, 29, 28])
    assert list(s.n) == [30, 29, 28] and s.block(0).shape == (30, 29)
    write_1e_files(tmp_path, "h", n=40, k=7, R=30.0, l_max=2, gauges=("v",))
    e1 = io.h5_read(tmp_path / "dat" / "h1.h5", "En", 29)
    np.testing.assert_allclose(e1, s.eig[30:59], atol=1e-12)
    d = io.h5_read(tmp_path / "dat" / "h12v.h5", "d_if", 29, 28)
    np.testing.assert_allclose(d, s.block(1), atol=1e-12)


def test_thomas_reiche_kuhn_sum_rule():
    """Sum over every p state of the basis of the 1s oscillator strengths is 1
    (one electron), in the length form 2 dE |<p|z|1s>|^2, the velocity form
    2 |<p|d/dz|1s>|^2 / dE and the mixed form 2 <p|z|1s><p|d/dz|1s>: z|1s> lies
    in the basis span, so the finite basis keeps the sum rule."""
    t, Es, Cs = solve_1e(n=60, k=9, R=40.0, Z=1.0, l_max=1)
    Dl = dipoles_1e(t, 9, Cs, 40.0, "l")[0][0, :]
    Dv = dipoles_1e(t, 9, Cs, 40.0, "v")[0][0, :]
    dE = Es[1] - Es[0][0]
    assert abs((2 * dE * Dl ** 2).sum() - 1.0) < 1e-10
    assert abs((2 * Dv ** 2 / dE).sum() - 1.0) < 1e-10
    assert abs((2 * Dl * Dv).sum() - 1.0) < 1e-10


def test_coupling_norm_is_the_dense_spectral_norm():
    """System.coupling_norm (power iteration on the blocks) against the
    dense 2-norm of the assembled coupling, both gauges."""
    from mpc_tdse.systems import random_system

    for g in "lv":
        s = random_system([30, 40, 25, 35], gauge=g, seed=1)
        off = s.offs
        C = np.zeros((s.ntot, s.ntot))
        for L in range(len(s.n) - 1):
            D = s.block(L)
            C[off[L]:off[L + 1], off[L + 1]:off[L + 2]] = D if g == "l" else -D
            C[off[L + 1]:off[L + 2], off[L]:off[L + 1]] = D.T
        assert abs(s.coupling_norm(iters=300) - np.linalg.norm(C, 2)) < 1e-9
