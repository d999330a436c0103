"""The 2e structure restatement (id2ec / r12 / d2e / w2e) against known
answers: Wigner symbols (closed forms and the 6j orthogonality relation),
the hydrogenic Slater integral F0(1s,1s) = 5Z/8, helium's s-limit and
sp-limit ground-state energies (-2.879028, -2.900516 a.u.; the reference's
own programs cannot be built here, so parity with them is unpinned), the
1 1S -> 2 1P oscillator strength in both gauges, and the file layout
`tdse -e 2` reads.
"""
import numpy as np
import pytest

from mpc_tdse import io
from mpc_tdse import structure2e as s2
from mpc_tdse.structure1e import solve_1e


def test_wigner_symbols():
    assert s2.wigner_3j0(1, 1, 0) == pytest.approx(-1 / np.sqrt(3), abs=1e-15)
    assert s2.wigner_3j0(2, 2, 2) == pytest.approx(-np.sqrt(2 / 35), abs=1e-15)
    assert s2.wigner_3j0(1, 1, 1) == 0.0 and s2.wigner_3j0(1, 2, 4) == 0.0
    assert s2.wigner_6j(1, 1, 1, 1, 1, 1) == pytest.approx(1 / 6, abs=1e-15)
    assert s2.wigner_6j(2, 2, 2, 2, 2, 2) == pytest.approx(-3 / 70, abs=1e-15)
    # sum_x (2x+1)(2f+1) {a b x; c d f}{a b x; c d g} = delta_fg (f, g allowed)
    for a, b, c, d in [(2, 1, 2, 1), (3, 2, 1, 2), (4, 4, 3, 2)]:
        for f in range(0, 7):
            for g in range(0, 7):
                v = sum((2 * x + 1) * (2 * f + 1) * s2.wigner_6j(a, b, x, c, d, f) *
                        s2.wigner_6j(a, b, x, c, d, g) for x in range(0, 12))
                ok = f == g and abs(a - d) <= f <= a + d and abs(b - c) <= f <= b + c
                assert abs(v - ok) < 1e-12, (a, b, c, d, f, g, v)


def test_cfg_files_round_trip(tmp_path):
    lines = s2.default_cfg_lines(1, 2, 3, 10)
    s2.write_cfg(tmp_path / "cfg-1.inp", 1, lines)
    assert s2.read_cfg(tmp_path / "cfg-1.inp", 1) == lines
    # natural parity only: p^2 cannot couple to L = 1, s-d cannot couple to L = 1
    with open(tmp_path / "bad.inp", "w") as f:
        f.write("1\n1 0\n3\n1 1 1 1 5\n1 0 2 1 5\n1 0 1 1 5\n")
    assert s2.read_cfg(tmp_path / "bad.inp", 1) == [(0, 0, 1, 0, 5)]
    idx = s2.config_index(lines)
    assert idx.shape[1] == 4 and len(idx) == sum(b - a for _, _, _, a, b in lines)


def test_hydrogenic_slater_integral():
    t, Es, Cs = solve_1e(60, 9, 40.0, 2.0, 0, 0.5, glq=15)
    rad = s2.Radial(t, 9, Cs, 40.0, 2)
    one = np.array([0])
    R = s2.slater_block(rad, 0, 0, one, 0, one, 0, one, 0, one)
    assert R.ravel()[0] == pytest.approx(5 * 2.0 / 8, abs=1e-6)


def test_helium_s_and_sp_limits_and_oscillator_strength():
    sys_s, ps = s2.helium(n=50, R=20.0, Z=2.0, l_max=0, L_max=0, n_inner=48, n_outer=48,
                          gauge="l", k_max="complete")
    assert ps["E_CI"][0][0] == pytest.approx(-2.879028, abs=2e-5)
    res = {}
    for g in ("l", "v"):
        sysm, p = s2.helium(n=50, R=20.0, Z=2.0, l_max=1, L_max=1, n_inner=48, n_outer=48,
                            gauge=g, k_max="complete")
        assert p["E_CI"][0][0] == pytest.approx(-2.900516, abs=3e-5)
        assert p["E_CI"][1][0] == pytest.approx(-2.1238, abs=2e-3)   # 2 1P
        dE = p["E_CI"][1][0] - p["E_CI"][0][0]
        z = p["D_CI"][0][0, 0]
        res[g] = 2 * dE * z * z if g == "l" else 2 * z * z / dE
        assert sysm.n.tolist() == [len(e) for e in p["E_CI"]]
    # f(1 1S -> 2 1P) = 0.276 exactly; the sp-limit CI gives ~0.26 in both gauges
    assert 0.25 < res["l"] < 0.28 and 0.25 < res["v"] < 0.28
    assert abs(res["l"] - res["v"]) < 0.03 * res["l"]


def test_v12_symmetric_and_reference_k_range():
    t, Es, Cs = solve_1e(40, 9, 20.0, 2.0, 2, 0.5, glq=15)
    rad = s2.Radial(t, 9, Cs, 20.0, 8)
    idx = s2.config_index(s2.default_cfg_lines(0, 2, 3, 8))
    Vr = s2.v12_matrix(0, idx, rad, "reference")
    Vc = s2.v12_matrix(0, idx, rad, "complete")
    assert np.array_equal(Vr, Vr.T)
    # the reference's k < l1max + l2max drops only the k = 4 multipole of d^2 pairs
    d2 = (idx[:, 1] == 2) & (idx[:, 3] == 2)
    diff = np.abs(Vr - Vc)
    assert diff[np.ix_(~d2, ~d2)].max() == 0.0
    assert 0.0 < diff.max() < 0.05 * np.abs(Vc).max()


def test_files_in_reference_layout(tmp_path):
    sysm, p = s2.helium(n=30, R=15.0, Z=2.0, l_max=1, L_max=1, n_inner=3, n_outer=12,
                        gauge="v")
    s2.write_2e_files(tmp_path, "he", p, "v")
    for L in range(2):
        E = io.h5_read(tmp_path / "dat" / f"heCI{L}.h5", "En_CI")
        assert np.array_equal(E, p["E_CI"][L])
        assert s2.read_cfg(tmp_path / "dat" / f"cfg-{L}.inp", L) == p["lines"][L]
    D = io.h5_read(tmp_path / "dat" / "heCI_01v.h5", "CI_dip")
    assert np.array_equal(D, p["D_CI"][0])
    # velocity-gauge CI dipoles couple the ground state to 1P states
    assert np.abs(D[0]).max() > 0.1


def test_outer_potential_is_summed_stably():
    """High box states of high l carry small-r noise that r^-(k+1) amplifies;
    the outer part of chi must be summed inwards, not as total minus a
    cumulative sum (which left R^6 of (5f,6f; 100f,100f) at -2e5 and a
    spurious CI state at -15 a.u.)."""
    t, Es, Cs = solve_1e(120, 9, 60.0, 2.0, 3, 0.5, glq=15)
    rad = s2.Radial(t, 9, Cs, 60.0, 100)
    a = np.array
    for k in (4, 5, 6):
        R = s2.slater_block(rad, k, 3, a([5]), 3, a([6]), 3, a([99]), 3, a([99]))[0, 0, 0, 0]
        assert abs(R) < 1e-2, (k, R)
