"""Python front end of libmpc_tdse.so (the C ABI in include/mpc_tdse.h).

Mirrors the reference's in-process interface for the propagation path:

* :class:`Context` holds what ``tdse::propV`` / ``tdse::propL`` receive --
  ``state_sz``, the per-block energies ``eig`` and the dipole blocks
  (src/tdse/include/tdse.hpp:66-101) -- resident on the GPU;
* :meth:`Context.rhs` is ``MatVecV/MatVecL::operator()``
  (src/tdse/tdse.cpp:14-73, :85-143);
* :meth:`Context.rk78_step` is one ``rkf.do_step`` (src/tdse/tdse.cpp:190);
* :meth:`Context.propagate` is the loop of ``propV``/``propL``
  (src/tdse/tdse.cpp:186-215), returning the coefficient vector and the
  per-step population / field / pre-renormalisation norm;
* :func:`pulse_setup`, :func:`to_au`, :func:`period`, :func:`field` are
  ``pulse::*Setup``, ``toAU``, ``period`` and the field functions
  (src/tdse/pulse.cpp).

All compute runs in the CUDA library; there is no CPU fallback.  Importing
works without a GPU (the library loads), but creating a context needs one.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .systems import System  # noqa: F401

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libmpc_tdse.so")
HEADER_PATH = os.path.join(os.path.dirname(os.path.dirname(_HERE)), "include", "mpc_tdse.h")

MPC_OK = 0
ERRORS = {-1: "MPC_ERR_ARG", -2: "MPC_ERR_CUDA", -3: "MPC_ERR_DEVICE", -4: "MPC_ERR_NOMEM",
          -5: "MPC_ERR_UNSTABLE"}
FIELD = {"sineEE": 0, "sineAA": 1, "sineAE": 2, "sineEA": 3, "gauss": 4}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class MpcError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Pulse(C.Structure):
    """``pulse::params`` plus the field function bound to it."""
    _fields_ = [("kind", C.c_int), ("Eo", C.c_double), ("w", C.c_double),
                ("cepd", C.c_double), ("a", C.c_double), ("b", C.c_double)]

    def as_array(self):
        return np.array([self.Eo, self.w, self.cepd, self.a, self.b])


_lib = None


def lib():
    """Loads libmpc_tdse.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} not built; run __graft_entry__.build() "
                          "(python -c 'import __graft_entry__ as g; g.build()')")
    L = C.CDLL(LIB_PATH)
    L.mpc_version.restype = C.c_int
    L.mpc_last_error.argtypes = [C.c_char_p, C.c_size_t]
    L.mpc_to_au.argtypes = [C.c_double, C.c_double, _dp, _dp]
    L.mpc_period.restype = C.c_double
    L.mpc_period.argtypes = [C.c_double, C.c_int]
    L.mpc_pulse_setup.argtypes = [C.c_int, C.c_char, C.c_double, C.c_double, C.c_double,
                                  C.c_int, C.c_double, C.POINTER(Pulse)]
    L.mpc_field.restype = C.c_double
    L.mpc_field.argtypes = [C.POINTER(Pulse), C.c_double]
    L.mpc_ctx_create.argtypes = [C.c_int, _ip, _dp, _dp, C.c_char, C.c_int, C.POINTER(C.c_void_p)]
    L.mpc_ctx_destroy.argtypes = [C.c_void_p]
    L.mpc_ctx_size.argtypes = [C.c_void_p]
    L.mpc_ctx_stream.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
    L.mpc_rhs.argtypes = [C.c_void_p, C.c_double, _dp, _dp]
    L.mpc_rk78_step.argtypes = [C.c_void_p, C.c_double, C.c_double, _dp]
    L.mpc_propagate.argtypes = [C.c_void_p, C.POINTER(Pulse), C.c_double, C.c_double, C.c_int,
                                C.c_int, _dp, _dp, _dp, _dp]
    L.mpc_state_set.argtypes = [C.c_void_p, _dp]
    L.mpc_state_get.argtypes = [C.c_void_p, _dp]
    L.mpc_advance.argtypes = [C.c_void_p, C.POINTER(Pulse), C.c_double, C.c_double, C.c_int,
                              C.c_int]
    L.mpc_history_get.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp]
    L.mpc_sync.argtypes = [C.c_void_p]
    L.mpc_profile_enable.argtypes = [C.c_void_p, C.c_int]
    L.mpc_profile_read.argtypes = [C.c_void_p, C.c_int, _dp, C.POINTER(C.c_longlong)]
    L.mpc_batch_rhs.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp]
    L.mpc_objective_threshold.argtypes = [C.c_void_p, C.c_double]
    L.mpc_batch_objective.argtypes = [C.c_void_p, C.c_int, C.POINTER(Pulse), C.c_int, _dp, _dp,
                                      C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, _dp,
                                      _dp]
    L.mpc_batch_objective_backward.argtypes = [C.c_void_p, _dp, _dp]
    L.mpc_batch_objective_info.argtypes = [C.c_void_p, _ip, _ip, _dp]
    L.mpc_batch_autotune.argtypes = [C.c_void_p, C.c_int, _dp, C.c_int]
    L.mpc_batch_fixed_plan.argtypes = [C.c_void_p, _dp, C.c_int]
    L.mpc_batch_propagate.argtypes = [C.c_void_p, C.c_int, C.POINTER(Pulse), _dp, _dp, C.c_double,
                                      C.c_double, C.c_double, C.c_double, C.c_int, _dp, _ip, _ip,
                                      _dp]
    L.mpc_propagate_batch.argtypes = L.mpc_batch_propagate.argtypes
    L.mpc_propagate_adaptive.argtypes = [C.c_void_p, C.POINTER(Pulse), C.c_double, C.c_double,
                                         C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
                                         _dp, _ip, _ip, _dp]
    L.mpc_probe_fp64_peak.argtypes = [C.c_int, _dp, _dp]
    L.mpc_pes.argtypes = [C.c_void_p, C.c_int, C.c_double, _dp, _dp, C.c_int, _dp]
    L.mpc_pes_summed.argtypes = [C.c_void_p, C.c_int, C.c_double, _dp, _dp, _dp, C.c_int]
    L.mpc_ctx_set_path.argtypes = [C.c_void_p, C.c_int]
    L.mpc_ctx_get_path.argtypes = [C.c_void_p]
    L.mpc_objective.argtypes = [C.c_void_p, C.POINTER(Pulse), C.c_int, _dp, C.c_double, C.c_double,
                                C.c_double, C.c_int, C.c_int, C.c_int, _dp, _dp]
    L.mpc_objective_backward.argtypes = [C.c_void_p, _dp, _dp]
    L.mpc_objective_gradient.argtypes = [C.c_void_p, C.POINTER(Pulse), C.c_int, _dp, C.c_double,
                                         C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, _dp,
                                         _dp, _dp, _dp]
    L.mpc_adjoint.argtypes = L.mpc_objective_gradient.argtypes
    L.mpc_launch_count.restype = C.c_longlong
    L.mpc_launch_count.argtypes = [C.c_void_p]
    L.mpc_batch_advance.argtypes = [C.c_void_p, C.c_int, C.POINTER(Pulse), _dp, C.c_double, _ip,
                                    C.c_int, _dp, _dp, _dp]
    L.mpc_ctx_set_wait_limit.argtypes = [C.c_void_p, C.c_double]
    L.mpc_ctx_inject_barrier_timeout.argtypes = [C.c_void_p]
    _lib = L
    return L


def last_error():
    buf = C.create_string_buffer(1024)
    lib().mpc_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def _check(rc):
    if rc != MPC_OK:
        raise MpcError(rc, last_error())


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_dp)


def _state(x):
    x = np.ascontiguousarray(x)
    if np.iscomplexobj(x):
        return np.ascontiguousarray(x, dtype=np.complex128).view(np.float64).copy()
    return np.ascontiguousarray(x, dtype=np.float64).copy()


def to_au(Io_Wcm2, w_eV):
    a, b = C.c_double(), C.c_double()
    _check(lib().mpc_to_au(Io_Wcm2, w_eV, C.byref(a), C.byref(b)))
    return a.value, b.value


def period(w_au, cycles):
    return lib().mpc_period(w_au, int(cycles))


def pulse_setup(shape, gauge, Io_au, w_au, cepd, cycles, tau=0.0):
    p = Pulse()
    shp = {"sine": 0, "gaussian": 1, 0: 0, 1: 1}[shape]
    _check(lib().mpc_pulse_setup(shp, gauge.encode(), Io_au, w_au, cepd, int(cycles), tau,
                                 C.byref(p)))
    return p


def field(p, t):
    return lib().mpc_field(C.byref(p), t)


def probe_fp64_peak(device=0):
    """(DMMA, DFMA) FP64 TFLOP/s of the device, measured."""
    a, b = C.c_double(), C.c_double()
    _check(lib().mpc_probe_fp64_peak(int(device), C.byref(a), C.byref(b)))
    return a.value, b.value


class Context:
    """A system resident on one GPU (``mpc_ctx``)."""

    def __init__(self, state_sz, eig, dip, gauge, device=0):
        L = lib()
        self.n = np.ascontiguousarray(state_sz, dtype=np.int32)
        self.gauge = gauge
        eig = np.ascontiguousarray(eig, dtype=np.float64)
        dip = np.ascontiguousarray(dip, dtype=np.float64)
        h = C.c_void_p()
        _check(L.mpc_ctx_create(len(self.n) - 1, self.n.ctypes.data_as(_ip), _ptr(eig), _ptr(dip),
                                gauge.encode(), int(device), C.byref(h)))
        self._h = h
        self.size = int(self.n.sum())

    @classmethod
    def from_system(cls, s, device=0):
        return cls(s.n, s.eig, s.dip, s.gauge, device)

    def close(self):
        if getattr(self, "_h", None):
            lib().mpc_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def stream(self):
        s = C.c_void_p()
        _check(lib().mpc_ctx_stream(self._h, C.byref(s)))
        return s.value

    def rhs(self, F, x):
        xf = _state(x)
        out = np.empty_like(xf)
        _check(lib().mpc_rhs(self._h, float(F), _ptr(xf), _ptr(out)))
        return out.view(np.complex128)

    def rk78_step(self, F, dt, x):
        xf = _state(x)
        _check(lib().mpc_rk78_step(self._h, float(F), float(dt), _ptr(xf)))
        return xf.view(np.complex128)

    def propagate(self, pulse, t0, dt, steps, x, pop_index=0, history=True):
        """Returns (ct, pop[steps+1], field[steps], norm[steps]) (history optional)."""
        xf = _state(x)
        pop = np.empty(steps + 1) if history else None
        fld = np.empty(max(steps, 1)) if history else None
        nrm = np.empty(max(steps, 1)) if history else None
        _check(lib().mpc_propagate(self._h, C.byref(pulse), float(t0), float(dt), int(steps),
                                   int(pop_index), _ptr(xf), _ptr(pop), _ptr(fld), _ptr(nrm)))
        ct = xf.view(np.complex128)
        if not history:
            return ct
        return ct, pop, fld[:steps], nrm[:steps]

    def propagate_into(self, pulse, t0, dt, steps, ct, pop=None, fld=None, nrm=None,
                       pop_index=0):
        """mpc_propagate on caller-owned float64 buffers (e.g. pinned host
        memory), in place and without copies: ct [2*size], pop [steps+1],
        fld [steps], nrm [steps]."""
        _check(lib().mpc_propagate(self._h, C.byref(pulse), float(t0), float(dt), int(steps),
                                   int(pop_index), _ptr(ct), _ptr(pop), _ptr(fld), _ptr(nrm)))

    # device-resident form
    def state_set(self, x):
        self._xbuf = _state(x)
        _check(lib().mpc_state_set(self._h, _ptr(self._xbuf)))

    def state_get(self):
        out = np.empty(2 * self.size)
        _check(lib().mpc_state_get(self._h, _ptr(out)))
        return out.view(np.complex128)

    def advance(self, pulse, t0, dt, steps, pop_index=0):
        _check(lib().mpc_advance(self._h, C.byref(pulse), float(t0), float(dt), int(steps),
                                 int(pop_index)))

    def history(self, steps):
        pop, fld, nrm = np.empty(steps + 1), np.empty(max(steps, 1)), np.empty(max(steps, 1))
        _check(lib().mpc_history_get(self._h, int(steps), _ptr(pop), _ptr(fld), _ptr(nrm)))
        return pop, fld[:steps], nrm[:steps]

    def sync(self):
        _check(lib().mpc_sync(self._h))

    # -- batched (many pulses) -------------------------------------------
    def batch_rhs(self, F, X):
        """dxdt for B states X [B, size] (complex) at fields F [B]."""
        X = np.ascontiguousarray(X, dtype=np.complex128)
        B = X.shape[0]
        F = np.ascontiguousarray(F, dtype=np.float64)
        xf = X.view(np.float64).reshape(B, -1).copy()
        out = np.empty_like(xf)
        _check(lib().mpc_batch_rhs(self._h, B, _ptr(F), _ptr(xf), _ptr(out)))
        return out.view(np.complex128).reshape(B, -1)

    def batch_autotune(self, B):
        """Tunes the batched GEMM tiles up to B pulses; returns rows of
        (pulses, tile width in real columns, pipeline depth, k split, us per RHS)."""
        cap = 32
        tab = np.zeros((cap, 5))
        r = lib().mpc_batch_autotune(self._h, int(B), _ptr(tab), cap)
        _check(min(r, 0))
        return [(int(a), int(b), int(c), int(d), float(e)) for a, b, c, d, e in tab[:r]]

    def batch_fixed_plan(self):
        """Rows of (pulses, kind, tile width, ring depth, us per step) chosen
        for the batched fixed step; kind 0: one cp.async-fed launch per
        Horner product, 1: one persistent launch, 2: one TMA-fed launch per
        product, 3: as 0 with each tile's coupled blocks in two CTAs."""
        cap = 32
        tab = np.zeros((cap, 5))
        r = lib().mpc_batch_fixed_plan(self._h, _ptr(tab), cap)
        _check(min(r, 0))
        return [(int(a), int(b), int(c), int(d), float(e)) for a, b, c, d, e in tab[:r]]

    def batch_propagate(self, pulses, t0, t_end, X, h0=0.05, dt_max=0.2, rtol=1e-10,
                        atol=1e-10, max_attempts=0):
        """Adaptive RKF78 of B pulses at once.  pulses: list of Pulse;
        t0, t_end: [B]; X: [B, size] complex start states.  Returns
        (X_final, accepted[B], rejected[B], t_final[B])."""
        B = len(pulses)
        arr = (Pulse * B)(*pulses)
        t0 = np.ascontiguousarray(np.broadcast_to(t0, (B,)), dtype=np.float64)
        t_end = np.ascontiguousarray(np.broadcast_to(t_end, (B,)), dtype=np.float64)
        xf = np.ascontiguousarray(X, dtype=np.complex128).view(np.float64).reshape(B, -1).copy()
        acc = np.zeros(B, dtype=np.int32)
        rej = np.zeros(B, dtype=np.int32)
        tf = np.zeros(B)
        _check(lib().mpc_batch_propagate(self._h, B, arr, _ptr(t0), _ptr(t_end), h0, dt_max, rtol,
                                         atol, int(max_attempts), _ptr(xf), acc.ctypes.data_as(_ip),
                                         rej.ctypes.data_as(_ip), _ptr(tf)))
        return xf.view(np.complex128).reshape(B, -1), acc, rej, tf

    def batch_advance(self, pulses, t0, dt, steps, X, pop_index=0, history=False):
        """Fixed-step propagation of B pulses at once with the reference's
        semantics (mpc_batch_advance).  pulses: list of Pulse; t0, steps: [B];
        X: [B, size] complex start states.  Returns X_final, or with
        history=True (X_final, pop [B, M+1], norm [B, M]), M = max(steps)."""
        B = len(pulses)
        arr = (Pulse * B)(*pulses)
        t0 = np.ascontiguousarray(np.broadcast_to(t0, (B,)), dtype=np.float64)
        st = np.ascontiguousarray(np.broadcast_to(steps, (B,)), dtype=np.int32)
        xf = np.ascontiguousarray(X, dtype=np.complex128).view(np.float64).reshape(B, -1).copy()
        M = int(st.max()) if B else 0
        pop = np.full((B, M + 1), np.nan) if history else None
        nrm = np.full((B, max(M, 1)), np.nan) if history else None
        _check(lib().mpc_batch_advance(self._h, B, arr, _ptr(t0), float(dt),
                                       st.ctypes.data_as(_ip), int(pop_index), _ptr(xf),
                                       _ptr(pop), _ptr(nrm)))
        Xf = xf.view(np.complex128).reshape(B, -1)
        if not history:
            return Xf
        return Xf, pop, nrm[:, :M]

    def propagate_adaptive(self, pulse, t0, t_end, x, h0=0.05, dt_max=0.2, rtol=1e-10,
                           atol=1e-10, max_attempts=0):
        """Adaptive RKF78 of one pulse (mpc_propagate_adaptive).  Returns
        (x_final, accepted, rejected, t_final)."""
        xf = _state(x).copy()
        acc, rej, tf = C.c_int(), C.c_int(), C.c_double()
        _check(lib().mpc_propagate_adaptive(self._h, C.byref(pulse), t0, t_end, h0, dt_max, rtol,
                                            atol, int(max_attempts), _ptr(xf), C.byref(acc),
                                            C.byref(rej), C.byref(tf)))
        return xf.view(np.complex128), acc.value, rej.value, tf.value

    # -- photoelectron spectrum ---------------------------------------------
    def pes(self, electrons=1, threshold=0.0, ct=None):
        """(pes [(L_max+1) x ngrid], {ground, norm, yield, excited}) of the
        current state (or of ct)."""
        ngrid = int(self.n.max())
        out = np.zeros((len(self.n), ngrid))
        st = np.zeros(4)
        cf = None if ct is None else _state(ct)
        _check(lib().mpc_pes(self._h, int(electrons), float(threshold), _ptr(cf), _ptr(out), ngrid,
                             _ptr(st)))
        return out, {"ground": st[0], "norm": st[1], "yield": st[2], "excited": st[3]}

    def pes_summed(self, electrons=1, threshold=0.0, ct=None):
        """(grid [n_1], pes [n_1]): the summed spectrum of `pes -s`."""
        n1 = int(self.n[1])
        grid, out = np.zeros(n1), np.zeros(n1)
        cf = None if ct is None else _state(ct)
        _check(lib().mpc_pes_summed(self._h, int(electrons), float(threshold), _ptr(cf),
                                    _ptr(grid), _ptr(out), n1))
        return grid, out

    # -- objective and adjoint gradient -------------------------------------
    def objective_threshold(self, thr):
        """Energy below which states count as not ionised in the yield
        objective (target < 0): J = 1 - sum_{E_i < thr} |c_i|^2 (default 0)."""
        _check(lib().mpc_objective_threshold(self._h, float(thr)))

    def objective(self, pulse, u, T, t0, dt, steps, x0, target=-1, ckpt_every=64):
        """Forward pass; J.  Keeps checkpoints for objective_backward."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        J = C.c_double()
        _check(lib().mpc_objective(self._h, C.byref(pulse), len(u), _ptr(u), float(T), float(t0),
                                   float(dt), int(steps), int(target), int(ckpt_every),
                                   _ptr(_state(x0)), C.byref(J)))
        self._adj_K, self._adj_steps = len(u), int(steps)
        return J.value

    def objective_backward(self):
        """(dJ/du [K], dJ/dF_n [steps]) of the last objective call."""
        g = np.zeros(self._adj_K)
        f = np.zeros(self._adj_steps)
        _check(lib().mpc_objective_backward(self._h, _ptr(g), _ptr(f)))
        return g, f

    def batch_objective(self, pulses, U, T, t0, dt, steps, X0, target=-1, ckpt_every=64):
        """Objective of B pulses at once (fixed step); U: [B, K] controls,
        T: [B] control windows; X0: [B, size] start states.  Returns J [B]
        and keeps checkpoints for batch_objective_backward."""
        B = len(pulses)
        arr = (Pulse * B)(*pulses)
        U = np.ascontiguousarray(np.asarray(U, dtype=np.float64).reshape(B, -1))
        K = U.shape[1]
        T = np.ascontiguousarray(np.broadcast_to(np.asarray(T, dtype=np.float64), (B,)))
        xf = np.ascontiguousarray(X0, dtype=np.complex128).view(np.float64).reshape(B, -1).copy()
        J = np.zeros(B)
        _check(lib().mpc_batch_objective(self._h, B, arr, K, _ptr(U) if K else None,
                                         _ptr(T) if K else None, float(t0), float(dt),
                                         int(steps), int(target), int(ckpt_every), _ptr(xf),
                                         _ptr(J)))
        self._badj = (B, K, int(steps))
        return J

    def batch_objective_info(self):
        """{ckpt_every, segments, device_bytes} of the last batch_objective."""
        k, n, b = C.c_int(), C.c_int(), C.c_double()
        _check(lib().mpc_batch_objective_info(self._h, C.byref(k), C.byref(n), C.byref(b)))
        return {"ckpt_every": k.value, "segments": n.value, "device_bytes": b.value}

    def batch_objective_backward(self):
        """(dJ/du [B, K], dJ/dF_n [B, steps]) of the last batch_objective."""
        B, K, steps = self._badj
        G = np.zeros((B, max(K, 1)))
        Fb = np.zeros((B, steps))
        _check(lib().mpc_batch_objective_backward(self._h, _ptr(G), _ptr(Fb)))
        return G[:, :K], Fb

    def batch_objective_gradient(self, pulses, U, T, t0, dt, steps, X0, target=-1,
                                 ckpt_every=64):
        J = self.batch_objective(pulses, U, T, t0, dt, steps, X0, target, ckpt_every)
        G, Fb = self.batch_objective_backward()
        return J, G, Fb

    def objective_gradient(self, pulse, u, T, t0, dt, steps, x0, target=-1, ckpt_every=64):
        J = self.objective(pulse, u, T, t0, dt, steps, x0, target, ckpt_every)
        g, f = self.objective_backward()
        return J, g, f

    KERNELS = {"rhs_stream": 0, "combine": 1, "renorm": 2, "batch_stage": 3, "batch_other": 4,
               "resident": 5}
    PATHS = {"auto": 0, "streaming": 1, "resident": 2}

    def set_path(self, path):
        _check(lib().mpc_ctx_set_path(self._h, self.PATHS.get(path, path)))

    @property
    def path(self):
        r = lib().mpc_ctx_get_path(self._h)
        if r < 0:
            _check(r)
        return {1: "streaming", 2: "resident"}[r]

    def set_wait_limit(self, seconds):
        """Bound on the persistent kernels' grid-barrier waits (default 2 s);
        a wait that runs out makes the call raise MpcError (MPC_ERR_DEVICE)."""
        _check(lib().mpc_ctx_set_wait_limit(self._h, float(seconds)))

    def inject_barrier_timeout(self):
        """Test hook: the next persistent launch gets a grid barrier that
        cannot complete, so its bounded wait runs out."""
        _check(lib().mpc_ctx_inject_barrier_timeout(self._h))

    def profile(self, on=True):
        _check(lib().mpc_profile_enable(self._h, int(bool(on))))

    def profile_read(self, kind):
        ms, n = C.c_double(), C.c_longlong()
        _check(lib().mpc_profile_read(self._h, self.KERNELS.get(kind, kind), C.byref(ms),
                                      C.byref(n)))
        return ms.value, n.value

    @property
    def launches(self):
        return int(lib().mpc_launch_count(self._h))
