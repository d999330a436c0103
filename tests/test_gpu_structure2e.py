"""The 2e structure restatement on the GPU and its inputs through the
propagation: the torch/GPU contractions and diagonalisation agree with the
numpy path; a genuine He CI system (states below 3 a.u.) propagates on the
GPU as the CPU oracle does; the `tdse -e 2` executable runs on the files it
writes.

Tolerances: CI energies 1e-10 relative, CI dipoles 1e-9 relative to their
largest entry (GEMM and eigensolver orders differ); populations 1e-9.
"""
import os
import subprocess

import numpy as np
import pytest

import mpc_tdse
from mpc_tdse import io
from mpc_tdse import structure2e as s2

pytestmark = pytest.mark.gpu

KW = dict(n=40, R=15.0, Z=2.0, l_max=1, L_max=2, n_inner=6, n_outer=30, gauge="v")


def test_device_path_matches_numpy():
    _, a = s2.helium(**KW)
    _, b = s2.helium(**KW, device="cuda")
    for L in range(3):
        assert np.max(np.abs(a["E_CI"][L] - b["E_CI"][L])) <= 1e-10 * np.max(np.abs(a["E_CI"][L]))
    for L in range(2):
        assert np.max(np.abs(a["D_CI"][L] - b["D_CI"][L])) <= 1e-9 * np.max(np.abs(a["D_CI"][L]))


def test_he_ci_propagation_matches_oracle(oracle):
    sysm, _ = s2.helium(**KW, e_cut=3.0)
    assert sysm.ntot > 50 and sysm.eig.min() < -2.8
    Io, w = mpc_tdse.to_au(5e14, 21.2)     # He resonance region
    tau = mpc_tdse.period(w, 3)
    p = mpc_tdse.pulse_setup("sine", "v", Io, w, 0.0, 3, tau)
    x0 = np.zeros(sysm.ntot, complex)
    x0[0] = 1.0
    steps = 300
    dt = tau / steps
    with mpc_tdse.Context.from_system(sysm) as ctx:
        ct, pop, fld, nrm = ctx.propagate(p, 0.0, dt, steps, x0)
    xo, popo, _, _ = oracle.propagate(sysm.n, sysm.eig, sysm.dip, "v", "sineAA", p.as_array(),
                                      0.0, dt, steps, x0)
    assert np.max(np.abs(np.abs(ct) ** 2 - np.abs(xo) ** 2)) < 1e-9
    assert 1.0 - np.abs(ct[0]) ** 2 > 1e-4      # the pulse does something


def test_cli_2e_on_restated_ci_files(tmp_path):
    sysm, parts = s2.helium(**KW, e_cut=3.0)
    s2.write_2e_files(tmp_path, "he", parts, "v")
    io.write_settings(tmp_path / "he.yaml", "he", 2, "v", sysm.n, 0.02, "sine", 21.2, 5e14, 2,
                      electrons=2)
    r = subprocess.run([io.TDSE, "-e", "2", "-f", "he.yaml", "-o", "out"], cwd=tmp_path,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    pop = np.loadtxt(tmp_path / "out" / "he_pop10.dat")
    Io, w = mpc_tdse.to_au(5e14, 21.2)
    tau = mpc_tdse.period(w, 2)
    p = mpc_tdse.pulse_setup("sine", "v", Io, w, 0.0, 2, tau)
    steps = int(tau / 0.02)
    x0 = np.zeros(sysm.ntot, complex)
    x0[0] = 1.0
    with mpc_tdse.Context.from_system(sysm) as ctx:
        _, pl, _, _ = ctx.propagate(p, 0.0, 0.02, steps, x0)
    assert len(pop) == steps + 1
    assert np.max(np.abs(pop[:, 1] - pl)) < 1e-12
    assert os.path.exists(tmp_path / "out" / "cfg-2.inp")
