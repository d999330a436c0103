"""Two-electron (He-like) CI structure inputs: the configuration index, the
electron-electron repulsion, the two-electron dipoles and the CI
diagonalisation that the reference's id2ec / r12 / d2e / w2e programs
produce, restated with numpy (optionally with torch on a GPU for the
Slater-integral contractions and the diagonalisation), so that genuine 2e
inputs for `tdse -e 2` exist without those programs.

Follows:
  * configuration files cfg-<L>.inp: header lines holding one integer are
    skipped, then "L S", the number of lines, and per line
    "n1 l1 l2 n2min n2max" (1-based n1, n2min; n2 runs n2min..n2max); lines
    whose (l1, l2) cannot couple to L with natural parity are dropped
    (cfg::readCfg, src/cfg_in.cpp:3-53);
  * configuration energies e = E_{n1 l1} + E_{n2 l2} in file order
    (genidx::saveIdx, src/id2ec/genidx.cpp:16-136);
  * V12 between singlet configurations (n1 l1 n2 l2; L):
      (-1)^{l1+l2} sqrt([l1][l1'][l2][l2']) sum_k
        [ (-1)^{L+l2+l1'} R^k(a b; c d) (l1 k l1')(l2 k l2') {l1' l2' L; l2 l1 k}
        + (-1)^{L+l1+l1'} R^k(a b; d c) (l1 k l2')(l2 k l1') {l1' l2' L; l1 l2 k} ]
    with the 3j symbols at zero projections, [l] = 2l + 1, each equivalent
    configuration (n1 l1 = n2 l2) scaled by 1/sqrt(2), and k running over
    0 <= k < l1max + l2max as the reference loops (k_max="complete" keeps
    k = l1max + l2max as well) (r_12::r12Glob, src/r12/r12.cpp:53-302);
  * Slater integrals R^k(a b; c d) = int dr1 P_a P_c(r1) chi(r1),
    chi(r1) = r1^-(k+1) int_0^r1 r^k P_b P_d + r1^k int_r1^R r^-(k+1) P_b P_d
    (intfn::fsltrLob, src/r12/integrator.cpp:49-131), here on Gauss-Legendre
    points per knot interval with Gauss-Legendre sub-rules between
    consecutive points for the cumulative inner integrals;
  * two-electron dipoles between L and L+1: the eight one-electron
    transition terms (electron 1 or 2, direct or swapped pairing, l up or
    down), each (-1)^phase sqrt(4 l^2 - 1)/sqrt(l) {l_a l_b L; L+1 1 l'}
    times the one-electron d1e block, the downward terms multiplied by -1 in
    the velocity gauge, 1/sqrt(2) per equivalent configuration and an overall
    (-1)^{L+1} sqrt(L+1) (dmx2e::genDipole, src/d2e/dmx2e.cpp:23-336);
  * H = diag(e) + V12, eigenpairs in ascending order (dsyevd), and the CI
    dipoles C_L^T T C_{L+1} (w2e::formCIh0 / formCIDipoles,
    src/w2e/w2e.cpp:17-124).
Wigner symbols are computed here from the Racah formulas with exact integer
arithmetic (the reference links a prebuilt library for them).
"""
from __future__ import annotations

import math
import os
from fractions import Fraction
from functools import lru_cache

import numpy as np

from .systems import System


# ---------------------------------------------------------------- Wigner symbols
@lru_cache(maxsize=None)
def wigner_3j0(a: int, b: int, c: int) -> float:
    """(a b c; 0 0 0) for integer a, b, c."""
    if a < 0 or b < 0 or c < 0 or c > a + b or c < abs(a - b):
        return 0.0
    J = a + b + c
    if J % 2:
        return 0.0
    g = J // 2
    f = math.factorial
    num = Fraction(f(J - 2 * a) * f(J - 2 * b) * f(J - 2 * c), f(J + 1))
    pre = Fraction(f(g), f(g - a) * f(g - b) * f(g - c))
    val = math.sqrt(num) * float(pre)
    return -val if g % 2 else val


def _tri(a, b, c):
    return c <= a + b and c >= abs(a - b)


@lru_cache(maxsize=None)
def wigner_6j(j1: int, j2: int, j3: int, j4: int, j5: int, j6: int) -> float:
    """{j1 j2 j3; j4 j5 j6} for integer arguments (Racah's single sum)."""
    if min(j1, j2, j3, j4, j5, j6) < 0:
        return 0.0
    if not (_tri(j1, j2, j3) and _tri(j1, j5, j6) and _tri(j4, j2, j6) and _tri(j4, j5, j3)):
        return 0.0
    f = math.factorial

    def delta(a, b, c):
        return Fraction(f(a + b - c) * f(a - b + c) * f(-a + b + c), f(a + b + c + 1))

    pre = delta(j1, j2, j3) * delta(j1, j5, j6) * delta(j4, j2, j6) * delta(j4, j5, j3)
    a1, a2, a3, a4 = j1 + j2 + j3, j1 + j5 + j6, j4 + j2 + j6, j4 + j5 + j3
    b1, b2, b3 = j1 + j2 + j4 + j5, j2 + j3 + j5 + j6, j3 + j1 + j6 + j4
    s = 0
    for t in range(max(a1, a2, a3, a4), min(b1, b2, b3) + 1):
        term = f(t + 1) // (f(t - a1) * f(t - a2) * f(t - a3) * f(t - a4) *
                            f(b1 - t) * f(b2 - t) * f(b3 - t))
        s += -term if t % 2 else term
    # sqrt of the exact prefactor, times the exact integer sum
    return math.sqrt(pre) * s


# ---------------------------------------------------------------- configurations
def read_cfg(path, L):
    """Lines (n1, l1, l2, n2min, n2max) of cfg-<L>.inp, 0-based n1 / n2min,
    n2max exclusive; invalid (l1, l2) for L dropped."""
    with open(path) as f:
        rows = [ln.split() for ln in f]
    it = iter(rows)
    for r in it:
        if len(r) != 1:
            break
    ncf = int(next(it)[0])
    out = []
    for r in it:
        if len(out) == ncf:
            break
        if not r:
            continue
        n1, l1, l2, n2a, n2b = (int(v) for v in r[:5])
        if abs(l1 - l2) <= L <= l1 + l2 and (L % 2) == ((l1 + l2) % 2):
            out.append((n1 - 1, l1, l2, n2a - 1, n2b))
    return out


def write_cfg(path, L, lines, S=0):
    """cfg-<L>.inp in the reference's layout (lines as read_cfg returns them)."""
    with open(path, "w") as f:
        f.write(f"{L}\n{L} {S}\n{len(lines)}\n")
        for n1, l1, l2, a, b in lines:
            f.write(f"{n1 + 1} {l1} {l2} {a + 1} {b}\n")


def default_cfg_lines(L, l_max, n_inner, n_outer):
    """Configurations n1 l1 n2 l2 (l1 <= l2, natural parity) with the inner
    electron in the lowest n_inner states of l1 and the outer one in states
    up to n_outer of l2 (n2 >= n1 when l1 == l2: each pair once)."""
    out = []
    for l1 in range(l_max + 1):
        for l2 in range(l1, l_max + 1):
            if not (abs(l1 - l2) <= L <= l1 + l2) or (L + l1 + l2) % 2:
                continue
            for n1 in range(n_inner):
                a = n1 if l1 == l2 else 0
                if a < n_outer:
                    out.append((n1, l1, l2, a, n_outer))
    return out


def config_index(lines):
    """[N, 4] int array of (n1, l1, n2, l2) in file order."""
    idx = [(n1, l1, n2, l2) for n1, l1, l2, a, b in lines for n2 in range(a, b)]
    return np.array(idx, dtype=np.int64).reshape(-1, 4)


# ---------------------------------------------------------------- radial functions
class Radial:
    """Bound / box 1e orbitals P_{nl}(r) on the Slater-integral grid: Gauss-
    Legendre points per knot interval (outer), and `m_inner` Gauss-Legendre
    points inside each gap between consecutive outer points (and [0, r_0],
    [r_last, R]) for the cumulative inner integrals."""

    def __init__(self, t, k, Cs, R, n_keep, glq=12, m_inner=4):
        from .structure1e import _basis

        gx, gw = np.polynomial.legendre.leggauss(glq)
        brk = np.unique(t)
        xs, ws = [], []
        for a, b in zip(brk[:-1], brk[1:]):
            xs.append(0.5 * (b - a) * gx + 0.5 * (b + a))
            ws.append(0.5 * (b - a) * gw)
        self.r = np.concatenate(xs)
        self.w = np.concatenate(ws)
        edges = np.concatenate([[0.0], self.r, [R]])
        ix, iw = np.polynomial.legendre.leggauss(m_inner)
        lo, hi = edges[:-1], edges[1:]
        self.ri = (0.5 * (hi - lo)[:, None] * ix[None, :] + 0.5 * (hi + lo)[:, None])
        self.wi = 0.5 * (hi - lo)[:, None] * iw[None, :]          # [ngap, m]
        Bo = _basis(t, k, self.r)
        Bi = _basis(t, k, self.ri.ravel())
        self.Po = [C[:n_keep].dot(Bo.T) for C in Cs]               # [n, q] per l
        self.Pi = [(C[:n_keep].dot(Bi.T)).reshape(n_keep, *self.ri.shape) for C in Cs]

    def chi(self, k, Pb, Pd, Pbi, Pdi, device=None):
        """chi^k(r) on the outer points for every pair (b, d): [nb, nd, q].
        device None: numpy; else a torch device (the arrays given as numpy)."""
        r, ri, wi = self.r, self.ri, self.wi
        wlo, whi = wi * ri ** k, wi * ri ** (-(k + 1.0))
        if device is None:
            lo = np.einsum("bgm,dgm,gm->bdg", Pbi, Pdi, wlo)    # int over each gap of r^k rho
            hi = np.einsum("bgm,dgm,gm->bdg", Pbi, Pdi, whi)
            cl = np.cumsum(lo, axis=-1)[..., :-1]                # int_0^{r_i}
            # int_{r_i}^R summed from R inwards: the r^-(k+1) weight makes the
            # innermost gaps large, and total - cumsum would cancel them away
            ch = np.flip(np.cumsum(np.flip(hi, -1), axis=-1), -1)[..., 1:]
            return cl * r ** (-(k + 1.0)) + ch * r ** k
        import torch

        t = lambda a: torch.as_tensor(a, dtype=torch.float64, device=device)  # noqa: E731
        Pbi_, Pdi_ = t(Pbi), t(Pdi)
        lo = torch.einsum("bgm,dgm,gm->bdg", Pbi_, Pdi_, t(wlo))
        hi = torch.einsum("bgm,dgm,gm->bdg", Pbi_, Pdi_, t(whi))
        cl = torch.cumsum(lo, dim=-1)[..., :-1]
        ch = torch.flip(torch.cumsum(torch.flip(hi, [-1]), dim=-1), [-1])[..., 1:]
        return cl * t(r ** (-(k + 1.0))) + ch * t(r ** k)


# bound on the elements of one chi chunk (pairs x gaps x inner points)
_CHUNK = 1 << 25


def slater_block(rad, k, la, na, lc, nc, lb, nb, ld, nd, device=None):
    """R^k(a b; c d) for a in states na of la, c in nc of lc (electron 1) and
    b, d likewise (electron 2): [len(na), len(nc), len(nb), len(nd)].  The
    chi potentials are built from whichever electron has fewer pairs (R^k is
    symmetric under exchanging the electrons: int rho_ac chi[rho_bd] =
    int rho_bd chi[rho_ac]); the contraction over the radial grid is one GEMM
    per pair of the other electron, or one GEMM over chunks of b (on `device`
    if given)."""
    if len(na) * len(nc) < len(nb) * len(nd):
        return _slater_from_electron1(rad, k, la, na, lc, nc, lb, nb, ld, nd, device)
    Pa, Pc = rad.Po[la][na], rad.Po[lc][nc]
    rho1 = (Pa[:, None, :] * Pc[None, :, :] * rad.w).reshape(len(na) * len(nc), -1)
    gm = rad.ri.size
    step = max(1, _CHUNK // max(1, len(nd) * gm))
    out = np.empty((len(na) * len(nc), len(nb), len(nd)))
    if device is not None:
        import torch

        rho1_t = torch.as_tensor(rho1, dtype=torch.float64, device=device)
    for b0 in range(0, len(nb), step):
        bs = nb[b0:b0 + step]
        X = rad.chi(k, rad.Po[lb][bs], rad.Po[ld][nd], rad.Pi[lb][bs], rad.Pi[ld][nd], device)
        if device is None:
            R = rho1 @ X.reshape(len(bs) * len(nd), -1).T
        else:
            R = (rho1_t @ X.reshape(len(bs) * len(nd), -1).T).cpu().numpy()
        out[:, b0:b0 + len(bs), :] = R.reshape(len(na) * len(nc), len(bs), len(nd))
    return out.reshape(len(na), len(nc), len(nb), len(nd))


def _slater_from_electron1(rad, k, la, na, lc, nc, lb, nb, ld, nd, device=None):
    """R^k(a b; c d) = sum_r w chi[rho_ac](r) P_b(r) P_d(r): the potentials of
    the (few) electron-1 pairs, then one [nb x q] x [q x nd] GEMM per pair."""
    X = rad.chi(k, rad.Po[la][na], rad.Po[lc][nc], rad.Pi[la][na], rad.Pi[lc][nc], device)
    Pb, Pd = rad.Po[lb][nb], rad.Po[ld][nd]
    nac = len(na) * len(nc)
    out = np.empty((nac, len(nb), len(nd)))
    if device is None:
        wX = X.reshape(nac, -1) * rad.w
        for i in range(nac):
            out[i] = (Pb * wX[i]) @ Pd.T
    else:
        import torch

        t = lambda a: torch.as_tensor(a, dtype=torch.float64, device=device)  # noqa: E731
        wX = X.reshape(nac, -1) * t(rad.w)
        Pb_t, Pd_t = t(Pb), t(Pd)
        for i in range(nac):
            out[i] = ((Pb_t * wX[i]) @ Pd_t.T).cpu().numpy()
    return out.reshape(len(na), len(nc), len(nb), len(nd))


# ---------------------------------------------------------------- matrices
def v12_matrix(L, idx, rad, k_max="reference", device=None, lmax12=None):
    """Dense symmetric electron-electron repulsion between the configurations
    idx [N, 4] (n1, l1, n2, l2) of total L.  lmax12: the largest l1 and l2 over
    the configurations of every L (the reference bounds k by their sum)."""
    N = len(idx)
    l1m, l2m = lmax12 if lmax12 else (int(idx[:, 1].max()), int(idx[:, 3].max()))
    kmax = l1m + l2m if k_max in ("reference", "complete") else int(k_max)
    kset = range(kmax + (1 if k_max == "complete" else 0))
    V = np.zeros((N, N))
    chans = {}
    for i, (n1, l1, n2, l2) in enumerate(idx):
        chans.setdefault((int(l1), int(l2)), []).append(i)
    for (l1, l2), I in chans.items():
        I = np.array(I)
        for (m1, m2), J in chans.items():
            J = np.array(J)
            yn = math.sqrt((2 * l1 + 1) * (2 * m1 + 1) * (2 * l2 + 1) * (2 * m2 + 1))
            sgn = -1.0 if (l1 + l2) % 2 else 1.0
            n1i, n2i = idx[I, 0], idx[I, 2]
            n1j, n2j = idx[J, 0], idx[J, 2]
            u1i, u2i, u1j, u2j = (np.unique(v) for v in (n1i, n2i, n1j, n2j))
            pos = lambda u, v: np.searchsorted(u, v)  # noqa: E731
            block = np.zeros((len(I), len(J)))
            for k in kset:
                # direct: electron 1 a->c (l1->m1), electron 2 b->d (l2->m2)
                if (wigner_3j0(l1, k, m1) != 0.0 and wigner_3j0(l2, k, m2) != 0.0 and
                        (L + l2 + m1) % 2 == (L + l1 + m2) % 2):
                    ang = ((-1.0) ** (L + l2 + m1) * wigner_3j0(l1, k, m1) *
                           wigner_3j0(l2, k, m2) * wigner_6j(m1, m2, L, l2, l1, k))
                    if ang != 0.0:
                        R = slater_block(rad, k, l1, u1i, m1, u1j, l2, u2i, m2, u2j, device)
                        block += ang * R[pos(u1i, n1i)[:, None], pos(u1j, n1j)[None, :],
                                         pos(u2i, n2i)[:, None], pos(u2j, n2j)[None, :]]
                # exchange: electron 1 a->d (l1->m2), electron 2 b->c (l2->m1)
                if (wigner_3j0(l1, k, m2) != 0.0 and wigner_3j0(l2, k, m1) != 0.0 and
                        (L + l1 + m1) % 2 == (L + l2 + m2) % 2):
                    ang = ((-1.0) ** (L + l1 + m1) * wigner_3j0(l1, k, m2) *
                           wigner_3j0(l2, k, m1) * wigner_6j(m1, m2, L, l1, l2, k))
                    if ang != 0.0:
                        R = slater_block(rad, k, l1, u1i, m2, u2j, l2, u2i, m1, u1j, device)
                        block += ang * R[pos(u1i, n1i)[:, None], pos(u2j, n2j)[None, :],
                                         pos(u2i, n2i)[:, None], pos(u1j, n1j)[None, :]]
            V[np.ix_(I, J)] = sgn * yn * block
    eq = (idx[:, 0] == idx[:, 2]) & (idx[:, 1] == idx[:, 3])
    s = np.where(eq, np.sqrt(0.5), 1.0)
    V *= s[:, None] * s[None, :]
    return 0.5 * (V + V.T)


def dipole_2e(Lf, idx_i, idx_f, D1e, gauge):
    """Two-electron dipole block [Ni, Nf] between the configurations of
    L = Lf - 1 and Lf.  D1e[l]: the d1e block between l and l+1.  Built per
    pair of channels (l1, l2) -> (l1', l2'): the angular conditions are
    scalars there, and each of the eight terms is a gather of one d1e block
    masked by the spectator electron's state."""
    Li = Lf - 1
    down = -1.0 if gauge == "v" else 1.0
    T = np.zeros((len(idx_i), len(idx_f)))

    def chans(idx):
        out = {}
        for q, (n1, l1, n2, l2) in enumerate(idx):
            out.setdefault((int(l1), int(l2)), []).append(q)
        return {k: np.array(v) for k, v in out.items()}

    ci, cf = chans(idx_i), chans(idx_f)
    for (l1i, l2i), I in ci.items():
        n1i, n2i = idx_i[I, 0], idx_i[I, 2]
        for (l1f, l2f), J in cf.items():
            n1f, n2f = idx_f[J, 0], idx_f[J, 2]
            blk = np.zeros((len(I), len(J)))
            # (moving l, its states, spectator l, its states, final l, final
            #  states, final spectator l, its states, phase exponent)
            for up, terms in ((True, ((l1i, n1i, l2i, n2i, l1f, n1f, l2f, n2f, l2i + l1f),
                                      (l2i, n2i, l1i, n1i, l2f, n2f, l1f, n1f, l1i + l2f),
                                      (l1i, n1i, l2i, n2i, l2f, n2f, l1f, n1f, l2i + l2f),
                                      (l2i, n2i, l1i, n1i, l1f, n1f, l2f, n2f, l1i + l1f))),
                              (False, ((l1i, n1i, l2i, n2i, l1f, n1f, l2f, n2f, l2i + l1i),
                                       (l2i, n2i, l1i, n1i, l2f, n2f, l1f, n1f, l1i + l2i),
                                       (l1i, n1i, l2i, n2i, l2f, n2f, l1f, n1f, l2i + l1i),
                                       (l2i, n2i, l1i, n1i, l1f, n1f, l2f, n2f, l1i + l2i)))):
                for la, na, lb, nb, lf, nf, lo, no, ph in terms:
                    if lb != lo or (la + 1 != lf if up else la - 1 != lf):
                        continue
                    lm = lf if up else la           # the larger l of the transition
                    six = wigner_6j(la, lb, Li, Lf, 1, lf)
                    if six == 0.0:
                        continue
                    amp = (-1.0) ** ph * math.sqrt(4.0 * lm * lm - 1.0) / math.sqrt(lm) * six
                    if up:
                        d = D1e[la][na[:, None], nf[None, :]]
                    else:
                        d = down * D1e[lf][nf[None, :], na[:, None]]
                    blk += np.where(nb[:, None] == no[None, :], amp * d, 0.0)
            T[np.ix_(I, J)] = blk
    eqi = (idx_i[:, 0] == idx_i[:, 2]) & (idx_i[:, 1] == idx_i[:, 3])
    eqf = (idx_f[:, 0] == idx_f[:, 2]) & (idx_f[:, 1] == idx_f[:, 3])
    T *= np.where(eqi, math.sqrt(0.5), 1.0)[:, None] * np.where(eqf, math.sqrt(0.5), 1.0)[None, :]
    return T * ((-1.0) ** Lf * math.sqrt(Lf))


def diagonalise(e2e, V, device=None):
    """Ascending CI energies and eigenvectors (columns) of diag(e) + V."""
    H = V + np.diag(e2e)
    if device is None:
        E, C = np.linalg.eigh(H)
    else:
        import torch

        Et, Ct = torch.linalg.eigh(torch.as_tensor(H, dtype=torch.float64, device=device))
        E, C = Et.cpu().numpy(), Ct.cpu().numpy()
    # sign convention (eigenvectors are defined up to sign): the largest
    # component of each is positive
    big = np.abs(C).argmax(axis=0)
    C = C * np.where(C[big, np.arange(C.shape[1])] < 0, -1.0, 1.0)[None, :]
    return E, C


# ---------------------------------------------------------------- driver
def helium(n=60, k=9, R=40.0, Z=2.0, l_max=2, L_max=2, n_inner=4, n_outer=20, gauge="v",
           k_max="reference", glq=12, m_inner=4, qsz=400, device=None, lines=None,
           e_cut=None):
    """He-like CI system for the propagation (System) and the intermediate
    arrays: 1e structure from the B-spline restatement, configurations from
    `lines[L]` (or default_cfg_lines), V12, 2e dipoles, CI diagonalisation.
    device: None (numpy) or a torch device for the Slater-integral
    contractions and the diagonalisation."""
    from .structure1e import dipoles_1e, solve_1e

    t, Es, Cs = solve_1e(n, k, R, Z, l_max, 0.5, glq=15)
    n_keep = max(n_outer, n_inner)
    rad = Radial(t, k, Cs, R, n_keep, glq=glq, m_inner=m_inner)
    D1e = dipoles_1e(t, k, Cs, R, gauge, qsz)
    lines = lines or [default_cfg_lines(L, l_max, n_inner, n_outer) for L in range(L_max + 1)]
    allx = np.concatenate([config_index(ln) for ln in lines])
    lmax12 = (int(allx[:, 1].max()), int(allx[:, 3].max()))
    idx, e2e, ECI, CCI = [], [], [], []
    for L in range(L_max + 1):
        ix = config_index(lines[L])
        e = np.array([Es[l1][n1] + Es[l2][n2] for n1, l1, n2, l2 in ix])
        V = v12_matrix(L, ix, rad, k_max, device, lmax12)
        E, C = diagonalise(e, V, device)
        idx.append(ix)
        e2e.append(e)
        ECI.append(E)
        CCI.append(C)
    T, Dci = [], []
    for L in range(L_max):
        TL = dipole_2e(L + 1, idx[L], idx[L + 1], D1e, gauge)
        T.append(TL)
        Dci.append(CCI[L].T @ TL @ CCI[L + 1])
    parts = {"lines": lines, "idx": idx, "e2e": e2e, "E_CI": ECI, "C_CI": CCI, "T": T,
             "D_CI": Dci, "E1": Es, "D1e": D1e}
    return system_from_parts(parts, gauge, e_cut, f"He-CI-{n}-R{int(R)}-l{l_max}"), parts


def system_from_parts(parts, gauge, e_cut=None, name="He-CI"):
    """The propagation System of the CI states (per L those below e_cut, as
    states_in_l selects the top-left blocks of the files)."""
    ECI, Dci = parts["E_CI"], parts["D_CI"]
    nst = [len(E) if e_cut is None else int(np.sum(E < e_cut)) for E in ECI]
    dip = [Dci[L][:nst[L], :nst[L + 1]].ravel() for L in range(len(Dci))]
    return System(nst, np.concatenate([E[:k] for E, k in zip(ECI, nst)]),
                  np.concatenate(dip) if dip else np.zeros(0), gauge, name)


def write_2e_files(root, pot, parts, gauge):
    """dat/<pot>CI<L>.h5 (En_CI, CI_vecs), dat/<pot>CI_<L><L+1><g>.h5 (CI_dip)
    and dat/cfg-<L>.inp in the reference's layout."""
    from . import io

    dat = os.path.join(root, "dat")
    os.makedirs(dat, exist_ok=True)
    for L, (E, C) in enumerate(zip(parts["E_CI"], parts["C_CI"])):
        io.h5_write(os.path.join(dat, f"{pot}CI{L}.h5"), {"En_CI": E, "CI_vecs": C})
        write_cfg(os.path.join(dat, f"cfg-{L}.inp"), L, parts["lines"][L])
    for L, D in enumerate(parts["D_CI"]):
        io.h5_write(os.path.join(dat, f"{pot}CI_{L}{L + 1}{gauge}.h5"), {"CI_dip": D})


def main(argv=None):
    """python -m mpc_tdse.structure2e: writes dat/ inputs for `tdse -e 2`
    (the reference's h1e/w1e/d1e + id2ec/r12/d2e/w2e sequence) and prints the
    time each stage took."""
    import argparse
    import time

    from .structure1e import write_1e_files

    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--out", default=".")
    ap.add_argument("--pot", default="he")
    ap.add_argument("--n", type=int, default=80, help="B-splines")
    ap.add_argument("--R", type=float, default=40.0, help="box radius (a.u.)")
    ap.add_argument("--Z", type=float, default=2.0)
    ap.add_argument("--lmax", type=int, default=2, help="largest 1e l")
    ap.add_argument("--Lmax", type=int, default=2, help="largest total L")
    ap.add_argument("--inner", type=int, default=8, help="inner-electron states per l")
    ap.add_argument("--outer", type=int, default=60, help="outer-electron states per l")
    ap.add_argument("--gauge", default="v", choices=["l", "v"])
    ap.add_argument("--k-max", default="reference")
    ap.add_argument("--device", default=None, help="torch device, e.g. cuda")
    a = ap.parse_args(argv)
    t0 = time.time()
    write_1e_files(a.out, a.pot, a.n, 9, a.R, a.Z, a.lmax, (a.gauge,))
    t1 = time.time()
    _, parts = helium(a.n, 9, a.R, a.Z, a.lmax, a.Lmax, a.inner, a.outer, a.gauge,
                      a.k_max if a.k_max in ("reference", "complete") else int(a.k_max),
                      device=a.device)
    t2 = time.time()
    write_2e_files(a.out, a.pot, parts, a.gauge)
    sizes = [len(E) for E in parts["E_CI"]]
    print(f"configurations per L: {sizes} (total {sum(sizes)})")
    print(f"ground state energy (a.u.): {parts['E_CI'][0][0]:.8f}")
    print(f"1e structure {t1 - t0:.2f} s, 2e CI (V12, dipoles, diagonalisation) {t2 - t1:.2f} s"
          f" on {a.device or 'cpu'}")


if __name__ == "__main__":
    main()
