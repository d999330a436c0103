"""Writes the golden fixtures in this folder from the reference's own code.

Run in a checkout where the reference source tree is present:
    make -f oracle/Makefile && python tests/golden/make_golden.py

Every number here comes from oracle/_ref/libref_tdse.so, i.e. the
reference's src/tdse/tdse.cpp (MatVecV / MatVecL, tdse::propV / propL) and
src/tdse/pulse.cpp compiled as they are, with only the missing third-party
pieces stood in (odeint's RKF78 step, a CBLAS).  Inputs are small seeded
synthetic systems in the reference's layout.
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "mp-citdse_b200"))

from oracle import Reference  # noqa: E402
from mpc_tdse.systems import hydrogen_like_1e, random_system  # noqa: E402


def main():
    ref = Reference()
    ref.use_plain_loops()
    out = {}
    # 1) single right-hand-side evaluations, ragged blocks
    for g in "lv":
        s = random_system([5, 7, 6, 4, 9], gauge=g, seed=11)
        rng = np.random.default_rng(12)
        x = rng.standard_normal(s.ntot) + 1j * rng.standard_normal(s.ntot)
        for F in (0.0, 0.37, -1.25):
            out[f"rhs_{g}_{F}"] = ref.rhs(s.n, s.eig, s.dip, g, F, x)
        out[f"rhs_{g}_n"], out[f"rhs_{g}_eig"], out[f"rhs_{g}_dip"] = s.n, s.eig, s.dip
        out[f"rhs_{g}_x"] = x
    np.savez_compressed(os.path.join(HERE, "rhs.npz"), **out)

    # 2) pulses: every shape/gauge, CEP 0 (as main) and CEP 0.3 (set-up path)
    out = {}
    ts = np.linspace(-5.0, 1200.0, 997)
    for shape in ("sine", "gaussian"):
        for g in "lv":
            for cepd in (0.0, 0.3):
                out[f"field_{shape}_{g}_{cepd}"] = np.array(
                    [ref.field(shape, g, 1e14, 1.5498, 10, t, cepd) for t in ts])
    out["t"] = ts
    out["steps_10cyc_800nm"] = np.array(ref.steps(1.5498, 10, 0.0, 0.1))
    out["steps_8cyc_390nm"] = np.array(ref.steps(3.179, 8, 0.0, 0.1))
    np.savez_compressed(os.path.join(HERE, "fields.npz"), **out)

    # 3) full reference-semantics propagations (tdse::propL / propV), 2 cycles
    out = {}
    for g, shape in (("l", "sine"), ("v", "sine"), ("l", "gaussian")):
        s = hydrogen_like_1e(40, 3, gauge=g, seed=5)
        x0 = np.zeros(s.ntot, complex)
        x0[0] = 1.0
        steps = ref.steps(1.5498, 2, 0.0, 0.1)
        with tempfile.TemporaryDirectory() as d:
            ct = ref.propagate(s.n, s.eig, s.dip, g, shape, 1e14, 1.5498, 2, 0.0, 0.1, steps,
                               x0, os.path.join(d, "h"), pop_n=0, pop_l=0)
            pop = np.loadtxt(os.path.join(d, "h_pop10.dat"))
            fld = np.loadtxt(os.path.join(d, "h_field.dat"))
            names = sorted(f for f in os.listdir(d) if "_ct_" in f)
        key = f"prop_{g}_{shape}"
        out[key + "_ct"] = ct
        out[key + "_pop"] = pop
        out[key + "_field"] = fld
        out[key + "_steps"] = np.array(steps)
        out[key + "_ctfiles"] = np.array(names)
        out[key + "_n"], out[key + "_eig"], out[key + "_dip"] = s.n, s.eig, s.dip
    np.savez_compressed(os.path.join(HERE, "propagate.npz"), **out)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
