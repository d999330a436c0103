"""Input files of the `tdse` drop-in: HDF5 datasets, the yaml settings and
the text coefficient files, in the reference's names and layouts.

* ``h5_write`` / ``h5_read`` / ``h5_dims`` wrap libmpc_host.so (the HDF5
  subset of host/h5lite.hpp: float64 datasets at the root group).
* ``write_inputs`` lays a ``System`` out the way the reference's main reads
  it (src/tdse/tdse_main.cpp:110-128, src/tdse/td_read.cpp:50-120):
  1e: ``dat/<pot><L>.h5:/En`` and ``dat/<pot><L><L+1><g>.h5:/d_if``;
  2e: ``dat/<pot>CI<L>.h5:/En_CI``, ``dat/<pot>CI_<L><L+1><g>.h5:/CI_dip``
  and ``dat/cfg-<L>.inp``.  Extra states (``pad``) can be appended so that
  the reader's top-left block selection is exercised.
* ``read_ct`` parses a ``<pot>_ct_<t>.dat`` file (src/tdse/tdse.cpp:150-157).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
HOSTLIB = os.path.join(os.path.dirname(_HERE), "lib", "libmpc_host.so")
TDSE = os.path.join(os.path.dirname(_HERE), "bin", "tdse")
_h = None


def _lib():
    global _h
    if _h is None:
        if not os.path.exists(HOSTLIB):
            raise ImportError(f"{HOSTLIB} not built")
        _h = C.CDLL(HOSTLIB)
        _h.mpc_h5_write.argtypes = [C.c_char_p, C.c_int, C.POINTER(C.c_char_p),
                                    C.POINTER(C.c_int), C.POINTER(C.c_longlong),
                                    C.POINTER(C.POINTER(C.c_double))]
        _h.mpc_h5_dims.argtypes = [C.c_char_p, C.c_char_p, C.POINTER(C.c_int),
                                   C.POINTER(C.c_longlong)]
        _h.mpc_h5_read_block.argtypes = [C.c_char_p, C.c_char_p, C.c_longlong, C.c_longlong,
                                         C.POINTER(C.c_double)]
        _h.mpc_host_last_error.argtypes = [C.c_char_p, C.c_size_t]
    return _h


def _err():
    b = C.create_string_buffer(512)
    _lib().mpc_host_last_error(b, 512)
    return b.value.decode()


def h5_write(path, datasets):
    """datasets: {name: float64 array (1-D or 2-D)}."""
    names = list(datasets)
    arrs = [np.ascontiguousarray(datasets[k], dtype=np.float64) for k in names]
    cn = (C.c_char_p * len(names))(*[n.encode() for n in names])
    ranks = (C.c_int * len(names))(*[a.ndim for a in arrs])
    dims = [d for a in arrs for d in a.shape]
    cd = (C.c_longlong * max(1, len(dims)))(*dims)
    ptrs = (C.POINTER(C.c_double) * len(names))(*[a.ctypes.data_as(C.POINTER(C.c_double))
                                                   for a in arrs])
    if _lib().mpc_h5_write(str(path).encode(), len(names), cn, ranks, cd, ptrs):
        raise OSError(_err())


def h5_dims(path, name):
    r = C.c_int()
    d = (C.c_longlong * 2)()
    if _lib().mpc_h5_dims(str(path).encode(), name.encode(), C.byref(r), d):
        raise OSError(_err())
    return tuple(d[i] for i in range(r.value))


def h5_read(path, name, rows=None, cols=None):
    dims = h5_dims(path, name)
    rows = dims[0] if rows is None else rows
    if len(dims) == 1:
        out = np.empty(rows)
        cols = 0
    else:
        cols = dims[1] if cols is None else cols
        out = np.empty((rows, cols))
    if _lib().mpc_h5_read_block(str(path).encode(), name.encode(), rows, cols,
                                out.ctypes.data_as(C.POINTER(C.c_double))):
        raise OSError(_err())
    return out


def write_inputs(root, system, pot, electrons=1, pad=0, seed=0):
    """Writes dat/ files for `system` under `root` (see module docstring)."""
    rng = np.random.default_rng(seed)
    dat = os.path.join(root, "dat")
    os.makedirs(dat, exist_ok=True)
    g = system.gauge
    n = [int(v) for v in system.n]
    stem_e = pot + ("CI" if electrons == 2 else "")
    stem_d = pot + ("CI_" if electrons == 2 else "")
    set_e = "En_CI" if electrons == 2 else "En"
    set_d = "CI_dip" if electrons == 2 else "d_if"
    off = system.offs
    for L in range(len(n)):
        e = system.eig[off[L]:off[L + 1]]
        if pad:
            e = np.concatenate([e, e[-1] + np.arange(1, pad + 1)])
        h5_write(os.path.join(dat, f"{stem_e}{L}.h5"), {set_e: e})
        if electrons == 2:
            with open(os.path.join(dat, f"cfg-{L}.inp"), "w") as f:
                f.write(f"    1\t    # symmetry\n    {L}    0  # L and m_max\n    0\n")
    for L in range(len(n) - 1):
        D = system.block(L)
        if pad:
            big = rng.standard_normal((n[L] + pad, n[L + 1] + pad))
            big[:n[L], :n[L + 1]] = D
            D = big
        h5_write(os.path.join(dat, f"{stem_d}{L}{L + 1}{g}.h5"), {set_d: D})


def write_settings(path, pot, L_max, gauge, states_in_l, dt, shape, w_eV, Io, cycles,
                   electrons=1, cepd=0.0):
    """A settings file with the keys the reference's readConfig uses."""
    lmax_line = f"  L_max: {L_max}\n" if electrons == 2 else ""
    basis_lmax = f"  l_max: {L_max}             # l <= l_max\n" if electrons == 1 else "  l_max: 7\n"
    text = (
        "# settings for the tdse propagation\n"
        "Global_Settings:\n"
        f"  potential: \"{pot}\"   # potential name\n"
        f"{lmax_line}"
        f"  gauge: '{gauge}'          # 'l' length / 'v' velocity\n"
        "Basis_Settings:\n"
        f"{basis_lmax}"
        "Propagator_Settings:\n"
        f"  states_in_l: [{', '.join(str(int(v)) for v in states_in_l)}]\n"
        f"  dt: {dt} # time step\n"
        "Field_Parameters:\n"
        f"  shape: \"{shape}\"\n"
        f"  w: {w_eV}\n"
        f"  Io: {Io:.6e}\n"
        f"  cepd: {cepd}\n"
        f"  cycles: {cycles}\n")
    with open(path, "w") as f:
        f.write(text)


def read_ct(path):
    """(index, complex coefficients) of a _ct_ file."""
    rows = np.loadtxt(path, comments="#")
    return rows[:, 0].astype(int), rows[:, 1] + 1j * rows[:, 2]
