"""Writes the golden fixtures in this folder from the reference's own code.

Run in a checkout where the reference source tree is present:
    make -f oracle/Makefile REF=<reference tree> && python tests/golden/make_golden.py
    python tests/golden/make_golden.py --long    # the benchmark-size pulses

Every number here comes from oracle/_ref/libref_tdse.so, i.e. the
reference's src/tdse/tdse.cpp (MatVecV / MatVecL, tdse::propV / propL) and
src/tdse/pulse.cpp compiled as they are, with only the missing third-party
pieces stood in (odeint's RKF78 step, a CBLAS), or (pes.npz) from
oracle/_ref/libref_pes.so, the reference's src/pes/pes.cpp compiled as it is
against in-memory stand-ins for its HDF5 and yaml libraries.  Inputs are small seeded
synthetic systems in the reference's layout, and (--long) the benchmark's
1e hydrogen system from the structure restatement:
  cfg0_h1e.npz   one whole 10-cycle 800 nm 1e14 W/cm^2 pulse (11,032 steps,
                 dt 0.1, length gauge) through tdse::propL: final populations,
                 the _pop column and the _field column;
  batch_h1e.npz  16 pulses drawn as the batched workload draws them
                 (seed 0: intensity log-uniform 1e13-5e14 W/cm^2, 400-1600
                 nm, 4-20 cycles; CEP 0, which is what the reference's main
                 passes), each a whole pulse through propL at dt 0.05: final
                 populations and every 100th entry of each _pop column.
Both also keep a fingerprint of the system (energies, per-block Frobenius
norms of the dipoles) so that a test can check that it rebuilt the same
system before comparing.
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

    # 4) photoelectron spectra: the reference's own pes::genPES1e / genPES2e
    #    (src/pes/pes.cpp) with -s, on seeded coefficients
    from oracle import ReferencePes

    rp = ReferencePes()
    out = {}
    rng = np.random.default_rng(21)
    s = hydrogen_like_1e(40, 3, gauge="l", seed=5)
    files = [np.concatenate([s.eig[s.offs[L]:s.offs[L + 1]],
                             s.eig[s.offs[L + 1] - 1] + np.arange(1, 5)]) for L in range(4)]
    ct = rng.standard_normal(s.ntot) + 1j * rng.standard_normal(s.ntot)
    ct /= np.linalg.norm(ct)
    r = rp.run(1, s.n, files, ct)
    out["e1_n"], out["e1_eig"], out["e1_ct"] = s.n, s.eig, ct
    for L, rows in enumerate(r["blocks"]):
        out[f"e1_block{L}"] = rows
    out["e1_summed"] = r["summed"]
    out["e1_printed"] = np.array([r["printed"]["ground state pop"], r["printed"]["norm"],
                                  r["printed"]["yield"]])
    # 2e: CI-like sorted energies per block, the He+ 1s threshold at -2
    n2 = [30, 40, 45, 50]
    eig2, files2 = [], []
    for L, nL in enumerate(n2):
        e = np.sort(rng.uniform(-2.9 + 0.3 * L, 3.0, nL + 3))
        files2.append(e)
        eig2.append(e[:nL])
    eig2 = np.concatenate(eig2)
    ct2 = rng.standard_normal(sum(n2)) + 1j * rng.standard_normal(sum(n2))
    ct2[0] *= 8.0
    ct2 /= np.linalg.norm(ct2)
    r = rp.run(2, n2, files2, ct2, e0_1e=-2.0)
    out["e2_n"], out["e2_eig"], out["e2_ct"] = np.array(n2), eig2, ct2
    out["e2_threshold"] = np.array(-2.0)
    for L, rows in enumerate(r["blocks"]):
        out[f"e2_block{L}"] = rows
    out["e2_summed"] = r["summed"]
    out["e2_printed"] = np.array([r["printed"]["ground state pop"], r["printed"]["norm"],
                                  r["printed"]["yield"], r["printed"]["excited population"]])
    np.savez_compressed(os.path.join(HERE, "pes.npz"), **out)
    print("golden fixtures written to", HERE)


def h1e_system():
    from mpc_tdse.structure1e import hydrogen

    return hydrogen(n=300, k=9, R=200.0, l_max=5, gauge="l", states=[292] * 6)


def fingerprint(s):
    return s.eig.copy(), np.array([np.linalg.norm(s.block(L)) for L in range(len(s.n) - 1)])


def batch_pulse_params(B=16, seed=0):
    """(Io W/cm^2, photon energy eV, cycles) of the first B pulses of the
    batched workload's seeded draw (the same generator calls as bench.py)."""
    rng = np.random.default_rng(seed)
    n_all = 256
    Io = 10 ** rng.uniform(13, np.log10(5e14), n_all)
    lam = rng.uniform(400, 1600, n_all)
    rng.uniform(0, 2 * np.pi, n_all)   # CEP draw (the reference's main uses 0)
    cyc = rng.integers(4, 21, n_all)
    return [(float(Io[i]), 1239.84198 / float(lam[i]), int(cyc[i])) for i in range(B)]


def _one_pulse(job):
    """One whole pulse through the reference's propL on a single host thread
    (run in a process pool)."""
    Io, w_eV, cycles, dt = job
    ref = Reference()
    ref.use_openblas(1)
    s = h1e_system()
    x0 = np.zeros(s.ntot, complex)
    x0[0] = 1.0
    steps = ref.steps(w_eV, cycles, 0.0, dt)
    with tempfile.TemporaryDirectory() as d:
        ct = ref.propagate(s.n, s.eig, s.dip, "l", "sine", Io, w_eV, cycles, 0.0, dt, steps,
                           x0, os.path.join(d, "h"))
        pop = np.loadtxt(os.path.join(d, "h_pop10.dat"))
        fld = np.loadtxt(os.path.join(d, "h_field.dat"))
    return steps, np.abs(ct) ** 2, pop, fld


def main_long():
    import multiprocessing as mp

    s = h1e_system()
    eig, dnorm = fingerprint(s)
    jobs = [(1e14, 1.5498, 10, 0.1)] + [(Io, w, c, 0.05) for Io, w, c in batch_pulse_params()]
    with mp.get_context("spawn").Pool(min(len(jobs), os.cpu_count() or 1)) as pool:
        res = pool.map(_one_pulse, jobs)
    steps, pops, pop, fld = res[0]
    np.savez_compressed(os.path.join(HERE, "cfg0_h1e.npz"), steps=np.array(steps), pops=pops,
                        pop=pop, field=fld, eig=eig, dnorm=dnorm,
                        pulse=np.array([1e14, 1.5498, 10, 0.1]))
    out = {"eig": eig, "dnorm": dnorm, "dt": np.array(0.05),
           "params": np.array([j[:3] for j in jobs[1:]])}
    for b, (steps, pops, pop, _) in enumerate(res[1:]):
        out[f"steps_{b}"] = np.array(steps)
        out[f"pops_{b}"] = pops
        idx = np.unique(np.concatenate([np.arange(0, steps + 1, 100), [steps]]))
        out[f"popidx_{b}"] = idx
        out[f"pop_{b}"] = pop[idx, 1]
    np.savez_compressed(os.path.join(HERE, "batch_h1e.npz"), **out)
    print("benchmark-size fixtures written to", HERE)


if __name__ == "__main__":
    if "--long" in sys.argv:
        main_long()
    else:
        main()
