"""Seeded synthetic angular-momentum-blocked systems.

The reference reads its H0 eigenenergies and dipole blocks from HDF5 files
written by its structure programs (1e: h1e/d1e, 2e: w2e/d2e; loaded by
``tdrd::readEnergies`` / ``tdrd::readDipoles``, src/tdse/td_read.cpp:50-120).
Those programs are not part of this library, so benchmarks and tests use
seeded synthetic systems with the same layout, sizes and value ranges:

* ``eig``: flat float64 [n_total], block L holding its ``n[L]`` energies in
  ascending order (as the eigen-solvers write them);
* ``dip``: the row-major ``[n[L] x n[L+1]]`` dipole blocks back to back
  (the layout ``readDipoles`` produces from the top-left hyperslab).

Spectra are capped so that ``dt * (max|E| + |F|*||D||)`` stays inside the
imaginary-axis stability interval of the RKF78 step (about 2.36) at dt = 0.1.
"""
from __future__ import annotations

import numpy as np

RK78_IMAG_STABILITY = 2.365  # |R(iy)| <= 1 for 0 <= y <= this (Fehlberg 7(8), 8th-order weights)


class System:
    """Blocked H0 + dipole couplings, in the reference's array layout."""

    def __init__(self, n, eig, dip, gauge, name=""):
        self.n = np.asarray(n, dtype=np.int32)
        self.eig = np.ascontiguousarray(eig, dtype=np.float64)
        self.dip = np.ascontiguousarray(dip, dtype=np.float64)
        self.gauge = gauge
        self.name = name
        if self.eig.size != int(self.n.sum()):
            raise ValueError("eig size does not match sum(n)")
        if self.dip.size != self.dip_size(self.n):
            raise ValueError("dip size does not match sum(n[L]*n[L+1])")

    @staticmethod
    def dip_size(n):
        n = np.asarray(n, dtype=np.int64)
        return int((n[:-1] * n[1:]).sum())

    @property
    def L_max(self):
        return len(self.n) - 1

    @property
    def ntot(self):
        return int(self.n.sum())

    @property
    def offs(self):
        return np.concatenate([[0], np.cumsum(self.n)]).astype(np.int64)

    def coupling_norm(self, iters=60, device=None, seed=0):
        """||C||_2 of the dipole coupling C (the symmetric block-tridiagonal
        matrix of the length gauge; the velocity gauge's antisymmetric one has
        the same singular values up to the signs of its blocks, so the same
        power iteration on C^T C bounds both), by power iteration; device: a
        torch device for large systems, or None (numpy).  With max|E| it
        bounds the generator's spectral radius, max|E| + |F| ||C||_2, the
        quantity an explicit RK step must keep inside its stability
        interval."""
        offs = self.offs
        nb = len(self.n) - 1
        if device is not None:
            import torch

            blocks = [torch.as_tensor(self.block(L), device=device) for L in range(nb)]
            x = torch.as_tensor(np.random.default_rng(seed).standard_normal(self.ntot),
                                device=device)
            cat = torch.cat
            norm = torch.linalg.norm
        else:
            blocks = [self.block(L) for L in range(nb)]
            x = np.random.default_rng(seed).standard_normal(self.ntot)
            cat = np.concatenate
            norm = np.linalg.norm

        def apply(v, s_lo, s_up):
            # block L of the result: s_lo D_{L-1}^T v_{L-1} + s_up D_L v_{L+1}
            parts = []
            for L in range(nb + 1):
                acc = 0.0
                if L > 0:
                    acc = acc + s_lo * (blocks[L - 1].T @ v[offs[L - 1]:offs[L]])
                if L < nb:
                    acc = acc + s_up * (blocks[L] @ v[offs[L + 1]:offs[L + 2]])
                parts.append(acc)
            return cat(parts)

        # C: (1, s); C^T: (s, 1), s = +1 (length) or -1 (velocity)
        s = 1.0 if self.gauge == "l" else -1.0
        lam = 0.0
        for _ in range(iters):
            x = x / norm(x)
            y = apply(apply(x, 1.0, s), s, 1.0)   # C^T C x
            lam = float(norm(y))
            x = y
        return float(np.sqrt(lam))

    def block(self, L):
        """Dipole block L as a [n_L, n_{L+1}] view."""
        o = int((self.n[:L].astype(np.int64) * self.n[1:L + 1]).sum())
        return self.dip[o:o + int(self.n[L]) * int(self.n[L + 1])].reshape(self.n[L], self.n[L + 1])

    def dense_generator(self, F):
        """Dense complex matrix M with dc/dt = M c (for small checks)."""
        N = self.ntot
        off = self.offs
        S = np.zeros((N, N))
        for L in range(self.L_max):
            D = self.block(L)
            a, b, c = off[L], off[L + 1], off[L + 2]
            if self.gauge == "l":
                S[a:b, b:c] = D
                S[b:c, a:b] = D.T
            else:
                S[a:b, b:c] = -D
                S[b:c, a:b] = D.T
        H0 = np.diag(self.eig)
        if self.gauge == "l":
            return -1j * (H0 + F * S)
        return -1j * H0 + F * S


def random_system(n, gauge="l", seed=0, e_max=10.0, d_scale=1.0, name="random"):
    """Small dense random system (tests)."""
    rng = np.random.default_rng(seed)
    n = np.asarray(n, dtype=np.int32)
    eig = np.concatenate([np.sort(rng.uniform(-1.0, e_max, int(k))) for k in n])
    dip = rng.standard_normal(System.dip_size(n)) * d_scale / np.sqrt(max(1, int(n.max())))
    return System(n, eig, dip, gauge, name)


def hydrogen_like_1e(n_per_l=298, l_max=5, R=200.0, Z=1.0, gauge="l", seed=0):
    """Hydrogen-like 1e system with the shapes of a 300-B-spline, R=200 basis.

    Per l: box-bound Rydberg levels -Z^2/(2 n^2) for n = l+1 .. while the
    orbital (~2 n^2/Z) fits in the box, then box-continuum levels
    (k pi / R)^2 / 2.  Dipole blocks follow a smooth envelope in the energy
    difference with seeded random signs and magnitudes (length gauge: r-like
    matrix elements; velocity gauge: p-like).
    """
    rng = np.random.default_rng(seed)
    n = np.full(l_max + 1, n_per_l, dtype=np.int32)
    eig_blocks = []
    for l in range(l_max + 1):
        nb = []
        nn = l + 1
        while 2.0 * nn * nn / Z < 0.5 * R and len(nb) < n_per_l // 4:
            nb.append(-Z * Z / (2.0 * nn * nn))
            nn += 1
        k = np.arange(1, n_per_l - len(nb) + 1, dtype=np.float64) + 0.5 * l
        cont = 0.5 * (k * np.pi / R) ** 2
        eig_blocks.append(np.sort(np.concatenate([np.array(nb), cont]))[:n_per_l])
    eig = np.concatenate(eig_blocks)
    dips = []
    for l in range(l_max):
        Ei = eig_blocks[l][:, None]
        Ej = eig_blocks[l + 1][None, :]
        env = 1.0 / (1.0 + 4.0 * np.abs(Ei - Ej)) / (1.0 + np.maximum(0, Ei) + np.maximum(0, Ej))
        mag = rng.standard_normal((n_per_l, n_per_l))
        amp = 2.0 if gauge == "l" else 0.5
        dips.append((amp * env * mag).ravel())
    return System(n, eig, np.concatenate(dips), gauge, f"H-like-1e-{n_per_l}x{l_max + 1}")


def helium_like_2e(n_per_L=(3983, 4411, 4702, 4904), gauge="v", seed=0, e_max=15.0):
    """He-CI-like 2e system with the shapes of a 400-B-spline, R=150 CI basis.

    Per total L: a ground/doubly-excited bound set below the He+ threshold
    (-2 a.u.), singly-ionised continuum up to 0 and a doubly-ionised region up
    to ``e_max``; dense real dipole blocks with a seeded Gaussian spread scaled
    so that the coupling norm is of order one atomic unit.
    """
    rng = np.random.default_rng(seed)
    n = np.asarray(n_per_L, dtype=np.int32)
    eig_blocks = []
    for L, k in enumerate(n):
        k = int(k)
        nb = max(8, k // 40)
        ns = k // 2
        nd = k - nb - ns
        bound = -2.0 - 0.9037 * np.exp(-np.arange(nb) / 3.0) * (1.0 if L == 0 else 0.75)
        single = np.sort(rng.uniform(-2.0, 0.0, ns))
        double = np.sort(e_max * rng.uniform(0.0, 1.0, nd) ** 1.5)
        eig_blocks.append(np.sort(np.concatenate([bound, single, double])))
    eig = np.concatenate(eig_blocks)
    dips = []
    for L in range(len(n) - 1):
        a, b = int(n[L]), int(n[L + 1])
        sig = 0.5 / np.sqrt(a + b)
        dips.append((rng.standard_normal(a * b) * sig))
    return System(n, eig, np.concatenate(dips), gauge, f"He-like-2e-{int(n.sum())}")
