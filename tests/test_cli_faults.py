"""Failure paths of the `tdse` drop-in on its input files, on the host.

The reference's readers stop on the same inputs: readConfig asserts that
states_in_l has L_max + 1 entries (src/tdse/td_read.cpp:21), and the H5Cpp
reads in readEnergies / readDipoles throw on a missing file, a file that is
not HDF5, a missing dataset or a hyperslab larger than the dataset
(src/tdse/td_read.cpp:75, :109).  Here each of those ends the executable
with a non-zero status and a message naming the problem, before any GPU work
(the inputs are read and checked before a device context is created), so
these tests run without a GPU.  A non-finite energy in the file is refused
by mpc_ctx_create's input check, also before any device call.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from mpc_tdse import io
from mpc_tdse.systems import hydrogen_like_1e

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture()
def inputs(tmp_path):
    if not os.path.exists(io.TDSE):
        pytest.skip("tdse executable not built")
    s = hydrogen_like_1e(40, 3, gauge="l", seed=5)
    io.write_inputs(tmp_path, s, "h", electrons=1, pad=4)
    shutil.copy(os.path.join(GOLDEN, "settings_1e.yaml"), tmp_path / "h.yaml")
    return tmp_path


def _run(cwd):
    return subprocess.run([io.TDSE, "-e", "1", "-f", "h.yaml", "-o", "out"], cwd=cwd,
                          capture_output=True, text=True, timeout=120)


def _fails_with(r, *words):
    assert r.returncode != 0
    msg = (r.stderr + r.stdout).lower()
    for w in words:
        assert w.lower() in msg, (w, r.stderr, r.stdout)


def test_missing_energy_file(inputs):
    os.remove(inputs / "dat" / "h2.h5")
    _fails_with(_run(inputs), "cannot open", "h2.h5")


def test_truncated_dipole_file(inputs):
    p = inputs / "dat" / "h12l.h5"
    data = p.read_bytes()
    p.write_bytes(data[: len(data) // 2])
    _fails_with(_run(inputs), "hdf5")


def test_not_an_hdf5_file(inputs):
    (inputs / "dat" / "h0.h5").write_bytes(b"these bytes are not an HDF5 file\n" * 40)
    _fails_with(_run(inputs), "superblock")


def test_dataset_smaller_than_states_in_l(inputs):
    # block 1 holds 44 energies; ask for 50
    txt = (inputs / "h.yaml").read_text().replace("[40,40,40,40]", "[40,50,40,40]")
    (inputs / "h.yaml").write_text(txt)
    _fails_with(_run(inputs), "fewer entries")


def test_dipole_block_smaller_than_states_in_l(inputs):
    # replace the 0-1 dipole file by one with too few columns
    io.h5_write(inputs / "dat" / "h01l.h5", {"d_if": np.ones((44, 20))})
    _fails_with(_run(inputs), "smaller than the requested block")


def test_wrong_dataset_name(inputs):
    io.h5_write(inputs / "dat" / "h3.h5", {"Energies": np.arange(44.0)})
    _fails_with(_run(inputs), "no dataset 'En'")


def test_states_in_l_length_must_match_l_max(inputs):
    txt = (inputs / "h.yaml").read_text().replace("[40,40,40,40]", "[40,40,40]")
    (inputs / "h.yaml").write_text(txt)
    _fails_with(_run(inputs), "states_in_l")


def test_non_finite_energy(inputs):
    e = io.h5_read(inputs / "dat" / "h1.h5", "En")
    e[3] = np.nan
    io.h5_write(inputs / "dat" / "h1.h5", {"En": e})
    _fails_with(_run(inputs), "non-finite energy")
