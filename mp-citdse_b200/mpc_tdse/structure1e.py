"""One-electron structure inputs for the propagation: the eigenenergies and
dipole blocks that the reference's h1e / w1e / d1e programs write, restated
with numpy / scipy so that realistic hydrogen-like inputs exist without those
programs.

Follows:
  * knot sequence: k zeros, then a linear grid par, 2 par, ..., with
    par = R / (n - k + 1), then k knots at R (bsp::genKnots, src/h1e/bsp_gsl.cpp:3-44,
    type 'l');
  * Hamiltonian in the n - 2 interior B-splines (the first and last are
    dropped, so P(0) = P(R) = 0): H = m <B'|B'> - <B|Z/r|B> + m l(l+1) <B|1/r^2|B>,
    overlap <B|B>, integrals by Gauss-Legendre with `glq` points per knot
    interval; generalized eigenproblem per l, ascending energies; each
    eigenvector's sign fixed so that P(r) > 0 near r = 0 (h1e::genCoeff,
    src/h1e/h1e.cpp:104-181);
  * P_nl(r) and dP/dr on a `qsz`-point Gauss-Legendre rule over [0, R]
    (w1e prOuter, src/w1e/w1e.cpp:73-119);
  * dipoles D[n1][n2] = k_l * t(n1 l, n2 l+1), k_l = sqrt((l+1)^2 /
    (4 (l+1)^2 - 1)), with t = sum_q w_q r_q P1 P2 (length) or
    sum_q w_q P1 (P2' + (l+1) P2 / r_q) (velocity) (dmx1e::genDipole,
    src/d1e/dmx1e.cpp:24-140; dmx_int::tlenGL / tvelGL, src/d1e/integrator.cpp:3-32).
Gauss-Legendre nodes come from numpy (Golub-Welsch), not from the
reference's vendored fastgl.
"""
from __future__ import annotations

import os

import numpy as np
import scipy.interpolate
import scipy.linalg

from .systems import System


def knots_linear(n, k, R):
    par = R / float(n - k + 1)
    inner = np.cumsum(np.full(n - k, par))
    return np.concatenate([np.zeros(k), inner, np.full(k, float(R))])


def _basis(t, k, x, deriv=0):
    """Values of all n = len(t) - k B-splines of order k (degree k-1) at x."""
    n = len(t) - k
    out = np.zeros((len(x), n))
    for i in range(n):
        c = np.zeros(n)
        c[i] = 1.0
        spl = scipy.interpolate.BSpline(t, c, k - 1, extrapolate=False)
        v = spl.derivative(deriv)(x) if deriv else spl(x)
        out[:, i] = np.nan_to_num(v)
    return out


def solve_1e(n=300, k=9, R=200.0, Z=1.0, l_max=5, mass=0.5, glq=15):
    """Energies E[l] (n-2,) and coefficients C[l] (n-2 states x n splines)."""
    t = knots_linear(n, k, R)
    gx, gw = np.polynomial.legendre.leggauss(glq)
    brk = np.unique(t)
    xs, ws = [], []
    for a, b in zip(brk[:-1], brk[1:]):
        xs.append(0.5 * (b - a) * gx + 0.5 * (b + a))
        ws.append(0.5 * (b - a) * gw)
    x = np.concatenate(xs)
    w = np.concatenate(ws)
    B = _basis(t, k, x)[:, 1:-1]
    dB = _basis(t, k, x, 1)[:, 1:-1]
    S = (B * w[:, None]).T @ B
    T = (dB * w[:, None]).T @ dB
    V = (B * (w * Z / x)[:, None]).T @ B
    C2 = (B * (w / x ** 2)[:, None]).T @ B
    Es, Cs = [], []
    xsmall = x[0]
    b0 = _basis(t, k, np.array([xsmall]))[0, 1:-1]
    for l in range(l_max + 1):
        H = mass * T - V + mass * l * (l + 1) * C2
        E, Cv = scipy.linalg.eigh(H, S)
        sgn = np.sign(b0 @ Cv)
        sgn[sgn == 0] = 1.0
        Cv = Cv * sgn[None, :]
        full = np.zeros((n - 2, n))
        full[:, 1:-1] = Cv.T
        Es.append(E)
        Cs.append(full)
    return t, Es, Cs


def dipoles_1e(t, k, Cs, R, gauge="l", qsz=600):
    """Dipole blocks [l][n1, n2] between l and l+1 (all n-2 states each)."""
    gx, gw = np.polynomial.legendre.leggauss(qsz)
    x = 0.5 * R * (gx + 1.0)
    w = 0.5 * R * gw
    B = _basis(t, k, x)
    dB = _basis(t, k, x, 1)
    P = [C @ B.T for C in Cs]      # [states, q]
    dP = [C @ dB.T for C in Cs]
    out = []
    for l in range(len(Cs) - 1):
        lp1 = l + 1
        kl = np.sqrt(lp1 * lp1 / (4.0 * lp1 * lp1 - 1.0))
        if gauge == "l":
            D = (P[l] * (w * x)[None, :]) @ P[lp1].T
        else:
            D = (P[l] * w[None, :]) @ (dP[lp1] + lp1 * P[lp1] / x[None, :]).T
        out.append(kl * D)
    return out


def hydrogen(n=300, k=9, R=200.0, Z=1.0, l_max=5, gauge="l", states=None, glq=15, qsz=600):
    """A System from the 1e structure restatement.  `states` (per l, default
    all n - 2) keeps the lowest states of each l, as states_in_l does."""
    t, Es, Cs = solve_1e(n, k, R, Z, l_max, 0.5, glq)
    Ds = dipoles_1e(t, k, Cs, R, gauge, qsz)
    nst = [n - 2] * (l_max + 1) if states is None else list(states)
    eig = np.concatenate([Es[l][:nst[l]] for l in range(l_max + 1)])
    dip = np.concatenate([Ds[l][:nst[l], :nst[l + 1]].ravel() for l in range(l_max)])
    return System(nst, eig, dip, gauge, f"H-1e-{n}-k{k}-R{int(R)}")


def write_1e_files(root, pot="h", n=300, k=9, R=200.0, Z=1.0, l_max=5, gauges=("l", "v"),
                   glq=15, qsz=600):
    """dat/<pot><l>.h5 (En [n-2], Coeff [n-2 x n], Knots) and
    dat/<pot><l><l+1><g>.h5 (d_if [n-2 x n-2]) in the reference's layout."""
    from . import io

    t, Es, Cs = solve_1e(n, k, R, Z, l_max, 0.5, glq)
    dat = os.path.join(root, "dat")
    os.makedirs(dat, exist_ok=True)
    for l in range(l_max + 1):
        io.h5_write(os.path.join(dat, f"{pot}{l}.h5"), {"En": Es[l], "Coeff": Cs[l], "Knots": t})
    for g in gauges:
        for l, D in enumerate(dipoles_1e(t, k, Cs, R, g, qsz)):
            io.h5_write(os.path.join(dat, f"{pot}{l}{l + 1}{g}.h5"), {"d_if": D})
    return t, Es
