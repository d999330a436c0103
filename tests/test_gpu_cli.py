"""The drop-in `tdse` executable against the reference's own propagation
code (oracle/_ref: src/tdse/tdse.cpp propL/propV and their file output) on
the same HDF5 inputs: the same output file names, the same _field.dat text,
populations within 1e-9 and the 6-digit _ct_ files within their precision.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

import mpc_tdse
from mpc_tdse import io
from mpc_tdse.systems import helium_like_2e, hydrogen_like_1e
from oracle import Reference

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _run(cwd, *args, stdin=None):
    return subprocess.run([io.TDSE, *args], cwd=cwd, capture_output=True, text=True,
                          input=stdin, timeout=600)


def _compare(out_dir, ref_dir, pot, pop_name):
    ours = sorted(f for f in os.listdir(out_dir) if f != "settings.yaml" and not f.startswith("cfg"))
    refs = sorted(os.listdir(ref_dir))
    assert ours == refs
    with open(os.path.join(out_dir, f"{pot}_field.dat")) as a, \
            open(os.path.join(ref_dir, f"{pot}_field.dat")) as b:
        assert a.read() == b.read()
    pa = np.loadtxt(os.path.join(out_dir, pop_name))
    pb = np.loadtxt(os.path.join(ref_dir, pop_name))
    assert np.array_equal(pa[:, 0], pb[:, 0])
    assert np.max(np.abs(pa[:, 1] - pb[:, 1])) < 1e-9
    for f in ours:
        if "_ct_" in f:
            _, ca = io.read_ct(os.path.join(out_dir, f))
            _, cb = io.read_ct(os.path.join(ref_dir, f))
            assert np.max(np.abs(ca - cb)) <= 2e-6 * max(1.0, np.max(np.abs(cb))), f


def test_cli_1e_matches_reference_files(tmp_path):
    if not Reference.available():
        pytest.skip("reference build not present")
    s = hydrogen_like_1e(40, 3, gauge="l", seed=5)
    io.write_inputs(tmp_path, s, "h", electrons=1, pad=4)
    shutil.copy(os.path.join(GOLDEN, "settings_1e.yaml"), tmp_path / "h.yaml")
    r = _run(tmp_path, "-e", "1", "-f", "h.yaml", "-o", "out", "-n", "1", "-l", "0")
    assert r.returncode == 0, r.stderr
    assert "Core Potential:                       h" in r.stdout
    ref = Reference()
    ref.use_plain_loops()
    os.makedirs(tmp_path / "ref")
    x0 = np.zeros(s.ntot, complex)
    x0[0] = 1.0
    steps = ref.steps(1.5498, 2, 0.0, 0.1)
    ref.propagate(s.n, s.eig, s.dip, "l", "sine", 1e14, 1.5498, 2, 0.0, 0.1, steps, x0,
                  str(tmp_path / "ref" / "h"))
    _compare(tmp_path / "out", tmp_path / "ref", "h", "h_pop10.dat")
    # settings copied; a second run into the same directory asks, and 'n' stops it
    assert (tmp_path / "out" / "settings.yaml").exists()
    r2 = _run(tmp_path, "-e", "1", "-f", "h.yaml", "-o", "out", stdin="n\n")
    assert r2.returncode != 0 and "Overwrite? [y/n]" in r2.stdout

    # restart from a checkpoint file (-s): t0 comes from the file name
    ckpt = sorted((f for f in os.listdir(tmp_path / "out") if "_ct_" in f),
                  key=lambda f: float(f.split("_ct_")[1][:-4]))[4]
    t0 = float(ckpt.split("_ct_")[1][:-4])
    r3 = _run(tmp_path, "-e", "1", "-f", "h.yaml", "-o", "out2", "-s", f"out/{ckpt}")
    assert r3.returncode == 0, r3.stderr
    _, c0 = io.read_ct(tmp_path / "out" / ckpt)
    os.makedirs(tmp_path / "ref2")
    tau = mpc_tdse.period(mpc_tdse.to_au(1e14, 1.5498)[1], 2)
    steps2 = int((tau - t0) / 0.1)
    ref.propagate(s.n, s.eig, s.dip, "l", "sine", 1e14, 1.5498, 2, t0, 0.1, steps2, c0,
                  str(tmp_path / "ref2" / "h"))
    _compare(tmp_path / "out2", tmp_path / "ref2", "h", "h_pop10.dat")


def test_cli_2e_velocity_gauge_matches_reference_files(tmp_path):
    if not Reference.available():
        pytest.skip("reference build not present")
    s = helium_like_2e((60, 70, 65), gauge="v", seed=3)
    io.write_inputs(tmp_path, s, "he", electrons=2, pad=2)
    io.write_settings(tmp_path / "he.yaml", "he", 2, "v", s.n, 0.1, "sine", 3.179, 5e14, 1,
                      electrons=2)
    r = _run(tmp_path, "-e", "2", "-f", "he.yaml", "-o", "out")
    assert r.returncode == 0, r.stderr
    assert sorted(f for f in os.listdir(tmp_path / "out") if f.startswith("cfg")) == \
        ["cfg-0.inp", "cfg-1.inp", "cfg-2.inp"]
    ref = Reference()
    ref.use_plain_loops()
    os.makedirs(tmp_path / "ref")
    x0 = np.zeros(s.ntot, complex)
    x0[0] = 1.0
    steps = ref.steps(3.179, 1, 0.0, 0.1)
    ref.propagate(s.n, s.eig, s.dip, "v", "sine", 5e14, 3.179, 1, 0.0, 0.1, steps, x0,
                  str(tmp_path / "ref" / "he"))
    _compare(tmp_path / "out", tmp_path / "ref", "he", "he_pop10.dat")


def test_cli_rejects_bad_arguments(tmp_path):
    r = _run(tmp_path, "-e", "3", "-f", "x.yaml", "-o", "out")
    assert r.returncode != 0 and "Invalid number of electrons" in r.stdout


def test_cli_full_precision_restart_is_bit_exact(tmp_path):
    """-p writes <pot>_ct_<t>.h5 next to every text dump; restarting from one
    (-s file.h5) continues bit for bit: every later dump equals the
    uninterrupted run's."""
    s = hydrogen_like_1e(40, 3, gauge="l", seed=5)
    io.write_inputs(tmp_path, s, "h", electrons=1, pad=4)
    shutil.copy(os.path.join(GOLDEN, "settings_1e.yaml"), tmp_path / "h.yaml")
    r = _run(tmp_path, "-e", "1", "-f", "h.yaml", "-o", "out", "-p")
    assert r.returncode == 0, r.stderr
    h5s = sorted((f for f in os.listdir(tmp_path / "out") if f.endswith(".h5")),
                 key=lambda f: float(f.split("_ct_")[1][:-3]))
    txt = [f for f in os.listdir(tmp_path / "out") if f.endswith(".dat") and "_ct_" in f]
    assert len(h5s) == len(txt) >= 10
    # the h5 dump holds the text dump's numbers at full precision
    _, c_txt = io.read_ct(tmp_path / "out" / h5s[3].replace(".h5", ".dat"))
    c_h5 = io.h5_read(tmp_path / "out" / h5s[3], "ct")
    assert c_h5.shape == (s.ntot, 2)
    assert np.max(np.abs(c_h5[:, 0] + 1j * c_h5[:, 1] - c_txt)) <= 1e-6
    r2 = _run(tmp_path, "-e", "1", "-f", "h.yaml", "-o", "out2", "-p", "-s", f"out/{h5s[3]}")
    assert r2.returncode == 0, r2.stderr
    # the restarted run dumps every tenth of its own (shorter) run: compare the
    # dumps both runs wrote, the final state among them
    later = sorted((f for f in os.listdir(tmp_path / "out2") if f.endswith(".h5")),
                   key=lambda f: float(f.split("_ct_")[1][:-3]))
    common = [f for f in later if f in h5s]
    assert h5s[3] in common and later[-1] == h5s[-1] and len(common) >= 2
    for f in common:
        a = io.h5_read(tmp_path / "out2" / f, "ct")
        b = io.h5_read(tmp_path / "out" / f, "ct")
        assert np.array_equal(a, b), f
        assert io.h5_read(tmp_path / "out2" / f, "t")[0] == io.h5_read(tmp_path / "out" / f, "t")[0]
