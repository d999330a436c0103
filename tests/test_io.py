"""Host I/O of the drop-in (no GPU): the HDF5 subset, checked against a file
written by the HDF5 library itself, and the yaml settings reader."""
import glob
import os

import numpy as np
import pytest

from mpc_tdse import io


def test_hdf5_roundtrip_and_top_left_blocks(tmp_path):
    a = np.random.default_rng(0).standard_normal((7, 9))
    e = np.linspace(-0.5, 3.0, 11)
    p = tmp_path / "x.h5"
    io.h5_write(p, {"d_if": a, "En": e})
    assert open(p, "rb").read(8) == b"\x89HDF\r\n\x1a\n"
    assert io.h5_dims(p, "d_if") == (7, 9) and io.h5_dims(p, "En") == (11,)
    assert np.array_equal(io.h5_read(p, "d_if"), a)
    assert np.array_equal(io.h5_read(p, "d_if", 4, 5), a[:4, :5])   # readDipoles' hyperslab
    assert np.array_equal(io.h5_read(p, "En", 6), e[:6])            # readEnergies' first n
    with pytest.raises(OSError):
        io.h5_read(p, "missing")
    with pytest.raises(OSError):
        io.h5_read(p, "d_if", 8, 2)


def test_hdf5_reader_on_a_file_written_by_libhdf5():
    """scipy ships a MATLAB v7.3 file (HDF5 written by the HDF5 library:
    512-byte user block, superblock v0, v1 object headers, layout v2) whose
    'testdouble' scipy can read from the v7.1 (non-HDF5) copy."""
    scipy_io = pytest.importorskip("scipy.io")
    d = os.path.join(os.path.dirname(scipy_io.__file__), "matlab", "tests", "data")
    h5f = os.path.join(d, "testhdf5_7.4_GLNX86.mat")
    ref = os.path.join(d, "testdouble_7.1_GLNX86.mat")
    if not (os.path.exists(h5f) and os.path.exists(ref)):
        pytest.skip("scipy test data not installed")
    got = io.h5_read(h5f, "testdouble").ravel()
    want = scipy_io.loadmat(ref)["testdouble"].ravel()
    assert np.array_equal(got, want)


def test_write_inputs_layout(tmp_path):
    from mpc_tdse.systems import random_system

    s = random_system([5, 6, 4], gauge="v", seed=1)
    io.write_inputs(tmp_path, s, "he", electrons=2, pad=3)
    names = sorted(os.path.basename(f) for f in glob.glob(str(tmp_path / "dat" / "*")))
    assert names == ["cfg-0.inp", "cfg-1.inp", "cfg-2.inp", "heCI0.h5", "heCI1.h5", "heCI2.h5",
                     "heCI_01v.h5", "heCI_12v.h5"]
    assert io.h5_dims(tmp_path / "dat" / "heCI_01v.h5", "CI_dip") == (8, 9)
    assert np.array_equal(io.h5_read(tmp_path / "dat" / "heCI_12v.h5", "CI_dip", 6, 4), s.block(1))
    assert np.array_equal(io.h5_read(tmp_path / "dat" / "heCI1.h5", "En_CI", 6),
                          s.eig[5:11])
