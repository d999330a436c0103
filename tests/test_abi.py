"""The C ABI library loads without a GPU and exports every declared symbol;
host-only entry points (units, pulses) match the oracle; argument errors are
reported, not crashed on."""
import ctypes as C
import re

import numpy as np
import pytest

import mpc_tdse


def declared_functions():
    text = open(mpc_tdse.HEADER_PATH).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mpc_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = mpc_tdse.lib()
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_units_and_pulses_match_oracle(oracle):
    Io, w = mpc_tdse.to_au(1e14, 1.5498)
    ev, wc = oracle.units()
    assert Io == 1e14 * wc and w == 1.5498 * ev
    assert mpc_tdse.period(w, 10) == oracle.period(w, 10)
    ts = np.linspace(-1, 1200, 301)
    for shape, g, kind in [("sine", "l", "sineEE"), ("sine", "v", "sineAA"),
                           ("gaussian", "l", "gauss"), ("gaussian", "v", "gauss")]:
        tau = mpc_tdse.period(w, 10)
        for cepd in (0.0, 0.7):
            p = mpc_tdse.pulse_setup(shape, g, Io, w, cepd, 10, tau)
            po = oracle.pulse_setup(shape, g, Io, w, cepd, 10, tau)
            np.testing.assert_array_equal(p.as_array(), po)
            got = np.array([mpc_tdse.field(p, t) for t in ts])
            want = np.array([oracle.field(kind, po, t) for t in ts])
            np.testing.assert_allclose(got, want, rtol=1e-13, atol=1e-18)


def test_argument_errors_are_reported():
    L = mpc_tdse.lib()
    with pytest.raises(mpc_tdse.MpcError) as e:
        mpc_tdse.pulse_setup("sine", "x", 1.0, 1.0, 0.0, 2)
    assert e.value.code == -1 and "gauge" in str(e.value)
    h = C.c_void_p()
    n = np.array([3, 3], dtype=np.int32)
    rc = L.mpc_ctx_create(0, n.ctypes.data_as(C.POINTER(C.c_int)), None, None, b"l", 0,
                          C.byref(h))
    assert rc == -1
    assert L.mpc_rhs(None, 0.0, None, None) == -1
