"""The CPU oracle against the reference's own code and against known answers.

Golden fixtures (tests/golden/*.npz) were produced by the reference's
src/tdse/tdse.cpp and pulse.cpp (see tests/golden/make_golden.py); the
known-answer tests pin what the reference has no tests for: the RKF78 tableau,
order-8 convergence, exact field-free evolution.
"""
import math
import os
import tempfile


import numpy as np
import pytest
import scipy.linalg

from mpc_tdse.systems import System, hydrogen_like_1e, random_system


# -- against the reference's own code (golden fixtures) ----------------------

@pytest.mark.parametrize("g", ["l", "v"])
def test_rhs_matches_reference_golden(oracle, golden, g):
    z = golden("rhs.npz")
    n, eig, dip, x = z[f"rhs_{g}_n"], z[f"rhs_{g}_eig"], z[f"rhs_{g}_dip"], z[f"rhs_{g}_x"]
    for F in (0.0, 0.37, -1.25):
        ref = z[f"rhs_{g}_{F}"]
        got = oracle.rhs(n, eig, dip, g, F, x)
        assert np.max(np.abs(got - ref)) <= 1e-14 * max(1.0, np.max(np.abs(ref)))


def test_fields_match_reference_golden(oracle, golden):
    z = golden("fields.npz")
    ev, wc = oracle.units()
    ts = z["t"]
    for shape in ("sine", "gaussian"):
        for g in "lv":
            for cepd in (0.0, 0.3):
                tau = oracle.period(1.5498 * ev, 10)
                p = oracle.pulse_setup(shape, g, 1e14 * wc, 1.5498 * ev, cepd, 10, tau)
                kind = "gauss" if shape == "gaussian" else ("sineEE" if g == "l" else "sineAA")
                got = np.array([oracle.field(kind, p, t) for t in ts])
                want = z[f"field_{shape}_{g}_{cepd}"]
                if cepd == 0.0:  # the reference's main always passes CEP 0
                    np.testing.assert_array_equal(got, want)
                else:  # w*t + cepd: the reference build contracts it to an FMA
                    np.testing.assert_allclose(got, want, rtol=1e-10, atol=1e-15)
    # step counts of the reference's main (tdse_main.cpp:162-163)
    assert int(z["steps_10cyc_800nm"]) == int(oracle.period(1.5498 * ev, 10) / 0.1)
    assert int(z["steps_8cyc_390nm"]) == int(oracle.period(3.179 * ev, 8) / 0.1)


@pytest.mark.parametrize("case", [("l", "sine"), ("v", "sine"), ("l", "gaussian")])
def test_propagation_matches_reference_golden(oracle, golden, case):
    g, shape = case
    z = golden("propagate.npz")
    key = f"prop_{g}_{shape}"
    n, eig, dip = z[key + "_n"], z[key + "_eig"], z[key + "_dip"]
    steps = int(z[key + "_steps"])
    ev, wc = oracle.units()
    tau = oracle.period(1.5498 * ev, 2)
    p = oracle.pulse_setup(shape, g, 1e14 * wc, 1.5498 * ev, 0.0, 2, tau)
    kind = "gauss" if shape == "gaussian" else ("sineEE" if g == "l" else "sineAA")
    x0 = np.zeros(int(np.sum(n)), complex)
    x0[0] = 1
    ct, pop, fld, nrm = oracle.propagate(n, eig, dip, g, kind, p, 0.0, 0.1, steps, x0)
    ref_ct = z[key + "_ct"]
    assert np.max(np.abs(np.abs(ct) ** 2 - np.abs(ref_ct) ** 2)) < 1e-12
    assert np.max(np.abs(ct - ref_ct)) < 1e-11
    # the reference's _pop file (16 digits) and _field file (6 digits)
    assert np.max(np.abs(z[key + "_pop"][:, 1] - pop)) < 1e-14
    np.testing.assert_allclose(z[key + "_field"][:, 1], fld, rtol=1e-5, atol=1e-12)
    np.testing.assert_allclose(z[key + "_pop"][1:, 0], 0.1 * np.arange(1, steps + 1), rtol=1e-9)


# -- known answers -----------------------------------------------------------

def test_tableau_linear_order_conditions(oracle):
    A, b8, b7, c = oracle.tableau()
    one = np.ones(13)
    assert np.allclose(A.sum(1), c, atol=1e-15)
    for k in range(8):  # b^T A^k 1 = 1/(k+1)!  for k < 8 (order 8)
        assert abs(b8 @ np.linalg.matrix_power(A, k) @ one - 1 / math.factorial(k + 1)) < 1e-14
    for k in range(7):
        assert abs(b7 @ np.linalg.matrix_power(A, k) @ one - 1 / math.factorial(k + 1)) < 1e-14
    # quadrature conditions b^T c^k = 1/(k+1) up to order 8
    for k in range(8):
        assert abs(b8 @ c ** k - 1 / (k + 1)) < 1e-14


def test_rhs_equals_dense_generator(oracle):
    for g in "lv":
        s = random_system([4, 6, 5, 3], gauge=g, seed=7)
        rng = np.random.default_rng(1)
        x = rng.standard_normal(s.ntot) + 1j * rng.standard_normal(s.ntot)
        got = oracle.rhs(s.n, s.eig, s.dip, g, 0.73, x)
        np.testing.assert_allclose(got, s.dense_generator(0.73) @ x, atol=1e-13)


def test_fixed_step_converges_at_order_8(oracle):
    s = random_system([3, 4, 3], gauge="l", seed=2, e_max=2.0)
    x0 = np.zeros(s.ntot, complex)
    x0[0] = 1
    F, T = 0.4, 4.0
    exact = scipy.linalg.expm(s.dense_generator(F) * T) @ x0
    errs = []
    for nsteps in (8, 16):
        x = x0.copy()
        for _ in range(nsteps):
            x = oracle.rk78_step(s.n, s.eig, s.dip, "l", F, T / nsteps, x)
        errs.append(np.max(np.abs(x - exact)))
    order = math.log2(errs[0] / errs[1])
    assert 7.5 < order < 9.5, (errs, order)


def test_field_free_evolution_is_the_stability_polynomial(oracle):
    """F = 0: each coefficient is multiplied by R(-i e dt) per step, then the
    state is renormalised."""
    s = random_system([6, 5, 7], gauge="l", seed=4, e_max=15.0)
    A, b8, _, _ = oracle.tableau()
    rng = np.random.default_rng(3)
    x0 = rng.standard_normal(s.ntot) + 1j * rng.standard_normal(s.ntot)
    x0 /= np.linalg.norm(x0)
    dt, steps = 0.1, 50
    z = -1j * s.eig * dt
    R = np.ones_like(z)
    for k in range(13):
        R = R + z ** (k + 1) * (b8 @ np.linalg.matrix_power(A, k) @ np.ones(13))
    x = x0.copy()
    for _ in range(steps):
        x = R * x
        x /= np.linalg.norm(x)
    p = np.zeros(5)
    p[0], p[1], p[3] = 0.0, 1.0, 1.0  # Eo = 0 -> F(t) = 0
    ct, pop, fld, nrm = oracle.propagate(s.n, s.eig, s.dip, "l", "sineEE", p, 0.0, dt, steps, x0)
    assert np.all(fld == 0.0)
    np.testing.assert_allclose(ct, x, atol=1e-13)


def test_adaptive_reaches_end_and_matches_fine_fixed_step(oracle):
    s = hydrogen_like_1e(30, 2, gauge="l", seed=1)
    ev, wc = oracle.units()
    tau = oracle.period(1.5498 * ev, 1)
    p = oracle.pulse_setup("sine", "l", 1e14 * wc, 1.5498 * ev, 0.0, 1, tau)
    x0 = np.zeros(s.ntot, complex)
    x0[0] = 1
    xa, st = oracle.propagate_adaptive(s.n, s.eig, s.dip, "l", "sineEE", p, 0.0, tau, 0.1, 1.0,
                                       1e-10, 1e-10, x0, field_mode=1)
    assert st["rc"] == 0 and st["t"] == tau and st["accepted"] > 0
    xb, st2 = oracle.propagate_adaptive(s.n, s.eig, s.dip, "l", "sineEE", p, 0.0, tau, 0.01,
                                        1.0, 1e-13, 1e-13, x0, field_mode=1)
    assert np.max(np.abs(np.abs(xa) ** 2 - np.abs(xb) ** 2)) < 1e-8


def test_control_perturbation_interpolates_samples(oracle):
    rng = np.random.default_rng(0)
    u = rng.standard_normal(33)
    T = 10.0
    g = T / 32
    for k in range(33):
        assert abs(oracle.control_eval(u, T, k * g) - u[k]) < 1e-12
    assert oracle.control_eval(u, T, -0.1) == 0.0 and oracle.control_eval(u, T, T + 0.1) == 0.0


@pytest.mark.parametrize("g", ["l", "v"])
@pytest.mark.parametrize("target", [-1, 3])
def test_oracle_adjoint_matches_its_own_central_differences(oracle, g, target):
    """The checker's discrete adjoint against central differences of the
    checker's own forward (h = 1e-6), on the CPU: the GPU adjoint is compared
    with this gradient, so it is pinned independently here (1e-6 relative)."""
    s = hydrogen_like_1e(12, 2, gauge=g, seed=4)
    ev, wc = oracle.units()
    w = 1.5498 * ev
    tau = oracle.period(w, 1)
    kind = "sineEE" if g == "l" else "sineAA"
    p = oracle.pulse_setup("sine", g, 2e14 * wc, w, 0.0, 1, tau)
    rng = np.random.default_rng(7)
    K, steps, dt = 16, 120, 0.1
    u = rng.standard_normal(K) * 0.01 * p[0]
    T = steps * dt
    x0 = np.zeros(s.ntot, complex)
    x0[0] = 1.0
    J, grad, _, _ = oracle.objective_gradient(s.n, s.eig, s.dip, g, kind, p, u, T, 0.0, dt,
                                              steps, x0, target)
    assert J == oracle.objective(s.n, s.eig, s.dip, g, kind, p, u, T, 0.0, dt, steps, x0, target)
    h = 1e-6
    for k in (1, 7, 12):
        up, um = u.copy(), u.copy()
        up[k] += h
        um[k] -= h
        fd = (oracle.objective(s.n, s.eig, s.dip, g, kind, p, up, T, 0.0, dt, steps, x0, target) -
              oracle.objective(s.n, s.eig, s.dip, g, kind, p, um, T, 0.0, dt, steps, x0, target)) \
            / (2 * h)
        assert abs(fd - grad[k]) <= 1e-6 * np.max(np.abs(grad)), (k, fd, grad[k])


def test_pes_restatement_known_answers():
    """The restated pes binning on hand-made spectra: a 1e state falls in the
    first l = 1 bin whose half-widths bracket it and adds |c|^2 * 2/(width);
    a 2e state above the threshold gives its own density |c|^2 * 2/(E+ - E-);
    the ground population, norm, yield and excited population follow."""
    from oracle import pes_reference

    # 1e: blocks l = 0, 1, 2 of 6, 6, 3 states; the l = 1 energies form the
    # grid, whose slots run over 1 <= k <= state_sz[0] - 2 as in the reference
    E0 = [-0.5, -0.125, 0.05, 0.3, 0.6, 0.8]
    E1 = [-0.25, -0.1, 0.1, 0.3, 0.5, 0.7]
    E2 = [-0.05, 0.31, 0.9]
    eig = np.array(E0 + E1 + E2)
    ct = np.zeros(15, complex)
    ct[0] = 0.5                   # ground state (never binned: loops start at 1)
    ct[3] = 0.4                   # l = 0, E = 0.3: bin k = 3 (E1[3], half-widths 0.1)
    ct[6 + 2] = 0.3j              # l = 1, E = 0.1: bin k = 2
    ct[12 + 1] = 0.2              # l = 2, E = 0.31: bin k = 3
    pes, ground, norm, yld, _ = pes_reference([6, 6, 3], eig, ct, electrons=1)
    assert ground == 0.25
    assert abs(norm - (0.25 + 0.16 + 0.09 + 0.04)) < 1e-15
    assert abs(pes[0, 3] - 0.16 * 2 / 0.4) < 1e-14
    assert abs(pes[1, 2] - 0.09 * 2 / 0.4) < 1e-14
    assert abs(pes[2, 3] - 0.04 * 2 / 0.4) < 1e-14
    assert np.count_nonzero(pes) == 3
    assert abs(yld - (0.16 + 0.09 + 0.04)) < 1e-15
    # 2e: one block, threshold -2; states 1..n-2 above it are densities
    eig2 = np.array([-2.9, -2.1, -1.9, -1.5, -1.0, -0.2])
    c2 = np.array([0.8, 0.1, 0.2, 0.3, 0.1, 0.5], dtype=complex)
    pes2, g2, n2, y2, exc2 = pes_reference([6], eig2, c2, electrons=2, threshold=-2.0)
    assert abs(g2 - 0.64) < 1e-15
    assert pes2[0, 1] == 0.0                                 # -2.1 is below the threshold
    assert abs(pes2[0, 2] - 0.04 * 2 / (-1.5 + 2.1)) < 1e-14
    assert abs(pes2[0, 4] - 0.01 * 2 / (-0.2 + 1.5)) < 1e-14
    assert pes2[0, 5] == 0.0                                 # the top state has no upper edge
    assert abs(y2 - (0.04 + 0.09 + 0.01)) < 1e-15
    assert abs(exc2 - (0.01 + 0.04 + 0.09 + 0.01)) < 1e-15


def test_frozen_field_step_is_the_degree_12_stability_polynomial(oracle):
    """With F frozen over a step the system is linear and autonomous, so one
    RKF78 step (8th-order solution) is R(hM) x with R(z) = sum_m G_m z^m,
    G_m = b8^T A^(m-1) 1: degree 12 (the z^13 coefficient vanishes).  The
    batched fixed-step path evaluates the step this way, by Horner's rule
    (12 products with M instead of 13 stage slopes); here the identity is
    checked against the stage form of the restatement."""
    from mpc_tdse.systems import random_system

    A, b8, _, _ = oracle.tableau()
    G = [1.0]
    v = np.ones(13)
    for _ in range(13):
        G.append(float(b8 @ v))
        v = A @ v
    assert G[13] == 0.0
    assert all(abs(G[m] - 1.0 / math.factorial(m)) <= 1e-14 * G[m] for m in range(9))
    for g in "lv":
        s = random_system([20, 25, 18], gauge=g, seed=2, e_max=6.0)
        rng = np.random.default_rng(3)
        x = rng.standard_normal(s.ntot) + 1j * rng.standard_normal(s.ntot)
        F, h = 0.31, 0.07
        want = oracle.rk78_step(s.n, s.eig, s.dip, g, F, h, x)

        def M(y):
            return oracle.rhs(s.n, s.eig, s.dip, g, F, y)

        hv = G[12] * x
        for m in range(11, -1, -1):
            hv = h * M(hv) + G[m] * x
        assert np.max(np.abs(hv - want)) < 1e-13
