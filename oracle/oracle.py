"""ctypes front end of the checker libraries -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  Two libraries sit behind it:

* ``liboracle_tdse.so`` -- the C restatement in ``oracle_tdse.c`` (reference
  RHS, fixed-step RKF78 loop with frozen field and renormalisation, pulses;
  plus the adaptive driver and control perturbation that the reference lacks).
* ``_ref/libref_tdse.so`` -- the reference's own ``src/tdse/tdse.cpp`` and
  ``pulse.cpp`` built against stand-in odeint/CBLAS headers (see Makefile).
  Present only where it was built (it needs the reference source tree at build
  time; the built file then travels with the repository).

Array conventions match the reference: ``eig`` is the flat concatenation of
the per-block energies, ``dip`` the back-to-back row-major ``[n_L x n_{L+1}]``
dipole blocks, states are interleaved complex128 (``numpy.complex128`` arrays
are accepted and viewed as float64 pairs).
"""
from __future__ import annotations

import ctypes as C
import os
import glob

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)

FIELD_KINDS = {"sineEE": 0, "sineAA": 1, "sineAE": 2, "sineEA": 3, "gauss": 4}


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def _as_f64(x):
    x = np.ascontiguousarray(x)
    if np.iscomplexobj(x):
        x = x.astype(np.complex128).view(np.float64)
    return np.ascontiguousarray(x, dtype=np.float64)


def _load(path):
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is not built (run `make -f oracle/Makefile`)")
    return C.CDLL(path)


class Oracle:
    """The C restatement."""

    def __init__(self, path=None):
        self.lib = _load(path or os.path.join(HERE, "liboracle_tdse.so"))
        L = self.lib
        L.orc_rhs.argtypes = [C.c_int, _ip, _dp, _dp, C.c_char, C.c_double, _dp, _dp]
        L.orc_rk78_step.argtypes = [C.c_int, _ip, _dp, _dp, C.c_char, C.c_double, C.c_double, _dp]
        L.orc_propagate.argtypes = [C.c_int, _ip, _dp, _dp, C.c_char, C.c_int, _dp,
                                    C.c_int, _dp, C.c_double, C.c_double, C.c_double,
                                    C.c_int, C.c_int, _dp, _dp, _dp, _dp]
        L.orc_propagate_adaptive.argtypes = [C.c_int, _ip, _dp, _dp, C.c_char, C.c_int, _dp,
                                             C.c_double, C.c_double, C.c_double, C.c_double,
                                             C.c_double, C.c_double, C.c_int, C.c_int, _dp, _dp]
        L.orc_field.restype = C.c_double
        L.orc_field.argtypes = [C.c_int, _dp, C.c_double]
        L.orc_pulse_setup.argtypes = [C.c_int, C.c_char, C.c_double, C.c_double,
                                      C.c_double, C.c_int, C.c_double, _dp]
        L.orc_period.restype = C.c_double
        L.orc_period.argtypes = [C.c_double, C.c_int]
        L.orc_units.argtypes = [_dp, _dp]
        L.orc_control_eval.restype = C.c_double
        L.orc_control_eval.argtypes = [C.c_int, _dp, C.c_double, C.c_double]
        L.orc_tableau.argtypes = [_dp, _dp, _dp, _dp]
        L.orc_use_blas.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_set_yield_threshold.argtypes = [C.c_double]
        L.orc_objective_gradient.argtypes = [C.c_int, _ip, _dp, _dp, C.c_char, C.c_int, _dp,
                                             C.c_int, _dp, C.c_double, C.c_double, C.c_double,
                                             C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp]
        L.orc_objective.argtypes = [C.c_int, _ip, _dp, _dp, C.c_char, C.c_int, _dp, C.c_int, _dp,
                                    C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, _dp,
                                    _dp]

    # -- system helpers -------------------------------------------------
    @staticmethod
    def _sys(n, eig, dip):
        n = np.ascontiguousarray(n, dtype=np.int32)
        return n, _as_f64(eig), _as_f64(dip)

    def rhs(self, n, eig, dip, gauge, F, x):
        n, eig, dip = self._sys(n, eig, dip)
        xf = _as_f64(x)
        out = np.empty_like(xf)
        rc = self.lib.orc_rhs(len(n) - 1, _i(n), _d(eig), _d(dip), gauge.encode(), F, _d(xf), _d(out))
        if rc:
            raise ValueError(f"orc_rhs rc={rc}")
        return out.view(np.complex128)

    def rk78_step(self, n, eig, dip, gauge, F, dt, x):
        n, eig, dip = self._sys(n, eig, dip)
        xf = _as_f64(x).copy()
        rc = self.lib.orc_rk78_step(len(n) - 1, _i(n), _d(eig), _d(dip), gauge.encode(), F, dt, _d(xf))
        if rc:
            raise ValueError(f"orc_rk78_step rc={rc}")
        return xf.view(np.complex128)

    def propagate(self, n, eig, dip, gauge, field_kind, pars, t0, dt, steps, x,
                  pop_index=0, control=None, control_T=0.0):
        """Reference-semantics loop.  Returns (x, pop[steps+1], field[steps], norm[steps])."""
        n, eig, dip = self._sys(n, eig, dip)
        xf = _as_f64(x).copy()
        pars = np.ascontiguousarray(pars, dtype=np.float64)
        pop = np.empty(steps + 1)
        fld = np.empty(max(steps, 1))
        nrm = np.empty(max(steps, 1))
        if control is None:
            K, u = 0, np.zeros(1)
        else:
            u = np.ascontiguousarray(control, dtype=np.float64)
            K = len(u)
        kind = FIELD_KINDS[field_kind] if isinstance(field_kind, str) else int(field_kind)
        rc = self.lib.orc_propagate(len(n) - 1, _i(n), _d(eig), _d(dip), gauge.encode(), kind,
                                    _d(pars), K, _d(u), control_T, t0, dt, steps, pop_index,
                                    _d(xf), _d(pop), _d(fld), _d(nrm))
        if rc:
            raise ValueError(f"orc_propagate rc={rc}")
        return xf.view(np.complex128), pop, fld[:steps], nrm[:steps]

    def propagate_adaptive(self, n, eig, dip, gauge, field_kind, pars, t0, t_end, h0,
                           dt_max, rtol, atol, x, field_mode=1, max_attempts=10_000_000):
        n, eig, dip = self._sys(n, eig, dip)
        xf = _as_f64(x).copy()
        pars = np.ascontiguousarray(pars, dtype=np.float64)
        stats = np.zeros(4)
        kind = FIELD_KINDS[field_kind] if isinstance(field_kind, str) else int(field_kind)
        rc = self.lib.orc_propagate_adaptive(len(n) - 1, _i(n), _d(eig), _d(dip), gauge.encode(),
                                             kind, _d(pars), t0, t_end, h0, dt_max, rtol, atol,
                                             field_mode, max_attempts, _d(xf), _d(stats))
        return xf.view(np.complex128), {"accepted": int(stats[0]), "rejected": int(stats[1]),
                                        "t": stats[2], "h": stats[3], "rc": rc}

    def objective_gradient(self, n, eig, dip, gauge, field_kind, pars, u, T, t0, dt, steps,
                           x0, target=-1):
        """(J, dJ/du [K], dJ/dF_n [steps], x_N) of the fixed-step propagation."""
        n, eig, dip = self._sys(n, eig, dip)
        u = np.ascontiguousarray(u, dtype=np.float64)
        x0f = _as_f64(x0)
        J = C.c_double()
        g = np.zeros(len(u))
        fb = np.zeros(steps)
        xN = np.zeros_like(x0f)
        kind = FIELD_KINDS[field_kind] if isinstance(field_kind, str) else int(field_kind)
        rc = self.lib.orc_objective_gradient(len(n) - 1, _i(n), _d(eig), _d(dip), gauge.encode(),
                                             kind, _d(np.ascontiguousarray(pars, dtype=np.float64)),
                                             len(u), _d(u), T, t0, dt, steps, target, _d(x0f),
                                             C.byref(J), _d(g), _d(fb), _d(xN))
        if rc:
            raise ValueError(f"orc_objective_gradient rc={rc}")
        return J.value, g, fb, xN.view(np.complex128)

    def yield_threshold(self, thr):
        """Energy below which states count as bound in the yield objective."""
        self.lib.orc_set_yield_threshold(float(thr))

    def objective(self, n, eig, dip, gauge, field_kind, pars, u, T, t0, dt, steps, x0, target=-1):
        n, eig, dip = self._sys(n, eig, dip)
        u = np.ascontiguousarray(u, dtype=np.float64)
        J = C.c_double()
        kind = FIELD_KINDS[field_kind] if isinstance(field_kind, str) else int(field_kind)
        rc = self.lib.orc_objective(len(n) - 1, _i(n), _d(eig), _d(dip), gauge.encode(), kind,
                                    _d(np.ascontiguousarray(pars, dtype=np.float64)), len(u), _d(u),
                                    T, t0, dt, steps, target, _d(_as_f64(x0)), C.byref(J))
        if rc:
            raise ValueError(f"orc_objective rc={rc}")
        return J.value

    def field(self, kind, pars, t):
        pars = np.ascontiguousarray(pars, dtype=np.float64)
        k = FIELD_KINDS[kind] if isinstance(kind, str) else int(kind)
        return self.lib.orc_field(k, _d(pars), t)

    def pulse_setup(self, shape, gauge, Io_au, w_au, cepd, cycles, tau):
        pars = np.zeros(5)
        self.lib.orc_pulse_setup(0 if shape == "sine" else 1, gauge.encode(), Io_au, w_au,
                                 cepd, cycles, tau, _d(pars))
        return pars

    def period(self, w_au, cycles):
        return self.lib.orc_period(w_au, cycles)

    def units(self):
        a, b = C.c_double(), C.c_double()
        self.lib.orc_units(C.byref(a), C.byref(b))
        return a.value, b.value

    def control_eval(self, u, T, t):
        u = np.ascontiguousarray(u, dtype=np.float64)
        return self.lib.orc_control_eval(len(u), _d(u), T, t)

    def tableau(self):
        A = np.zeros((13, 13)); b8 = np.zeros(13); b7 = np.zeros(13); c = np.zeros(13)
        self.lib.orc_tableau(_d(A), _d(b8), _d(b7), _d(c))
        return A, b8, b7, c

    def use_openblas(self, threads=0):
        """Route the oracle's dgemv/dznrm2 through scipy's bundled OpenBLAS."""
        path = openblas_path()
        if path is None:
            return False
        h = C.CDLL(path)
        if threads > 0 and hasattr(h, "scipy_openblas_set_num_threads"):
            h.scipy_openblas_set_num_threads(C.c_int(threads))
        self._blas = h
        self.lib.orc_use_blas(C.cast(h.scipy_cblas_dgemv, C.c_void_p),
                              C.cast(h.scipy_cblas_dznrm2, C.c_void_p))
        return True

    def use_plain_loops(self):
        self.lib.orc_use_blas(None, None)


def openblas_path():
    try:
        import scipy
    except ImportError:
        return None
    d = os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs")
    c = sorted(glob.glob(os.path.join(d, "libscipy_openblas*.so")))
    return c[0] if c else None


class Reference:
    """The reference's own tdse.cpp / pulse.cpp (built by oracle/Makefile)."""

    PATH = os.path.join(HERE, "_ref", "libref_tdse.so")

    def __init__(self, path=None):
        self.lib = _load(path or self.PATH)
        L = self.lib
        L.ref_rhs.argtypes = [C.c_int, _ip, _dp, _dp, C.c_char, C.c_double, _dp, _dp]
        L.ref_propagate.argtypes = [C.c_int, _ip, _dp, _dp, C.c_char, C.c_int, C.c_double,
                                    C.c_double, C.c_int, C.c_double, C.c_double, C.c_int,
                                    C.c_int, C.c_int, C.c_char_p, _dp]
        L.ref_field.restype = C.c_double
        L.ref_field.argtypes = [C.c_int, C.c_char, C.c_double, C.c_double, C.c_int,
                                C.c_double, C.c_double]
        L.ref_steps.argtypes = [C.c_double, C.c_int, C.c_double, C.c_double]
        L.ref_set_blas.argtypes = [C.c_char_p, C.c_int]

    @classmethod
    def available(cls):
        return os.path.exists(cls.PATH)

    def use_openblas(self, threads=0):
        p = openblas_path()
        if p is None:
            return False
        return self.lib.ref_set_blas(p.encode(), int(threads)) == 0

    def use_plain_loops(self):
        self.lib.ref_set_blas(None, 0)

    def rhs(self, n, eig, dip, gauge, F, x):
        n = np.ascontiguousarray(n, dtype=np.int32)
        eig, dip, xf = _as_f64(eig), _as_f64(dip), _as_f64(x)
        out = np.empty_like(xf)
        self.lib.ref_rhs(len(n) - 1, _i(n), _d(eig), _d(dip), gauge.encode(), F, _d(xf), _d(out))
        return out.view(np.complex128)

    def steps(self, w_eV, cycles, t0, dt):
        return self.lib.ref_steps(w_eV, cycles, t0, dt)

    def field(self, shape, gauge, Io_W, w_eV, cycles, t, cepd=0.0):
        return self.lib.ref_field(0 if shape == "sine" else 1, gauge.encode(), Io_W, w_eV,
                                  cycles, cepd, t)

    def propagate(self, n, eig, dip, gauge, shape, Io_W, w_eV, cycles, t0, dt, steps, x,
                  prefix, pop_n=0, pop_l=0):
        n = np.ascontiguousarray(n, dtype=np.int32)
        eig, dip = _as_f64(eig), _as_f64(dip)
        xf = _as_f64(x).copy()
        rc = self.lib.ref_propagate(len(n) - 1, _i(n), _d(eig), _d(dip), gauge.encode(),
                                    0 if shape == "sine" else 1, Io_W, w_eV, cycles, t0, dt,
                                    steps, pop_n, pop_l, prefix.encode(), _d(xf))
        if rc:
            raise ValueError(f"ref_propagate rc={rc}")
        return xf.view(np.complex128)


class ReferencePes:
    """The reference's own src/pes/pes.cpp (genPES1e / genPES2e), built by
    oracle/Makefile against in-memory stand-ins for its HDF5 and yaml
    libraries."""

    PATH = os.path.join(HERE, "_ref", "libref_pes.so")

    def __init__(self, path=None):
        self.lib = _load(path or self.PATH)
        self.lib.ref_pes.argtypes = [C.c_int, C.c_int, C.c_int, _ip, _ip, _dp, C.c_double, _dp,
                                     C.c_char_p, C.c_char_p, C.c_size_t]

    @classmethod
    def available(cls):
        return os.path.exists(cls.PATH)

    def run(self, electrons, n, file_eig, ct, e0_1e=0.0, summed=True):
        """Runs genPES1e / genPES2e on `ct` with the block energies
        `file_eig` (a list of per-block arrays, each at least n[L] long: the
        files' full contents).  Returns {"blocks": [rows of each
        <prefix>_pes<L>.dat], "summed": rows of <prefix>_pes.dat (or None),
        "printed": {name: value}} -- the reference's own outputs."""
        import tempfile

        n = np.ascontiguousarray(n, dtype=np.int32)
        fsz = np.array([len(e) for e in file_eig], dtype=np.int32)
        fe = np.ascontiguousarray(np.concatenate(file_eig), dtype=np.float64)
        cf = _as_f64(ct).copy()
        buf = C.create_string_buffer(4096)
        with tempfile.TemporaryDirectory() as d:
            prefix = os.path.join(d, "out")
            rc = self.lib.ref_pes(int(electrons), int(bool(summed)), len(n) - 1, _i(n), _i(fsz),
                                  _d(fe), float(e0_1e), _d(cf), prefix.encode(), buf, 4096)
            text = buf.value.decode()
            if rc:
                raise ValueError(f"ref_pes: {text}")

            def rows(path):
                if not os.path.exists(path) or os.path.getsize(path) == 0:
                    return np.zeros((0, 2))
                return np.loadtxt(path, ndmin=2)

            blocks = [rows(f"{prefix}_pes{L}.dat") for L in range(len(n))]
            summed_rows = rows(f"{prefix}_pes.dat") if summed else None
        printed = {}
        for line in text.splitlines():
            if ":" in line:
                k, v = line.split(":", 1)
                printed[k.strip()] = float(v)
        return {"blocks": blocks, "summed": summed_rows, "printed": printed}


def pes_reference(n, eig, ct, electrons=1, threshold=0.0):
    """pes::genPES1e / genPES2e (src/pes/pes.cpp:48-262) restated with the
    same loops and first-match bins, on full-precision coefficients.
    Returns (pes [(L_max+1) x max(n)], ground, norm, yield, excited)."""
    n = [int(v) for v in n]
    offs = np.concatenate([[0], np.cumsum(n)])
    c2 = np.abs(np.asarray(ct)) ** 2
    ngrid = max(n)
    pes = np.zeros((len(n), ngrid))
    ion_yield = 0.0
    exc = 0.0
    if electrons == 1:
        E1 = eig[offs[1]:offs[2]]
        for l in range(len(n)):
            for i in range(1, n[l]):
                for k in range(1, n[0] - 1):
                    nd = abs(E1[k] - E1[k - 1])
                    pd = abs(E1[k + 1] - E1[k])
                    e = eig[offs[l] + i]
                    if E1[k] - 0.5 * nd < e < E1[k] + 0.5 * pd:
                        pes[l, k] += c2[offs[l] + i] * 2.0 / (nd + pd)
                        ion_yield += (E1[k] > 0) * c2[offs[l] + i]
                        break
    else:
        for L in range(len(n)):
            o = offs[L]
            for i in range(1, n[L] - 1):
                e = eig[o + i]
                if e - threshold > 0.0:
                    pes[L, i] = c2[o + i] * 2.0 / (eig[o + i + 1] - eig[o + i - 1])
                    ion_yield += c2[o + i]
                if o + i > 0:
                    exc += c2[o + i]
    return pes, c2[0], c2.sum(), ion_yield, exc


def pes_summed_reference(n, eig, ct, electrons=1, threshold=0.0):
    """The summed spectrum of `pes -s` restated: genPES1e adds the blocks'
    binned spectra per bin (src/pes/pes.cpp:127-137); genPES2e bins every
    state i >= 1 of every block onto the L = 1 energies, first matching bin
    k in 1 .. n_1 - 1, whose upper neighbour for k = n_1 - 1 is the first
    energy of L = 2 as the reference indexes its concatenated energies
    (src/pes/pes.cpp:215-245).  Returns (grid [n_1], pes [n_1]): grid holds
    E1[k] (1e) or E1[k] - threshold (2e); the reference writes the rows
    0 <= k <= n_1 - 2 (1e: n_0 - 2) whose grid energy is positive."""
    n = [int(v) for v in n]
    offs = np.concatenate([[0], np.cumsum(n)])
    c2 = np.abs(np.asarray(ct)) ** 2
    E1 = np.asarray(eig[offs[1]:offs[2]], dtype=np.float64)
    n1 = n[1]
    out = np.zeros(n1)
    if electrons == 1:
        per_l, _, _, _, _ = pes_reference(n, eig, ct, 1)
        for l in range(len(n)):
            for k in range(1, n[0] - 1):
                out[k] += per_l[l, k]
        return E1.copy(), out
    kmax = n1 - 1 if len(n) > 2 else n1 - 2
    for L in range(len(n)):
        for i in range(1, n[L]):
            e = eig[offs[L] + i]
            for k in range(1, kmax + 1):
                nd = abs(E1[k] - E1[k - 1])
                pd = abs(eig[offs[1] + k + 1] - E1[k])
                if E1[k] - 0.5 * nd < e < E1[k] + 0.5 * pd:
                    out[k] += c2[offs[L] + i] * 2.0 / (nd + pd)
                    break
    return E1 - threshold, out
