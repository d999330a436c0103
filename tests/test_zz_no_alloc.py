"""mpc_rhs_noalloc: the right-hand side for callers that cannot allocate
device memory (a framework whose caching allocator owns the GPU, a plugin
that may not allocate after start-up, a time-critical loop).  The caller
hands in device buffers it already owns; the library's only scratch is a
static 16 MiB device array.

Checked through the C ABI against the context entry point mpc_rhs, within
the tolerance of the other single-RHS tests (1e-13 relative), on two calls
in a row per system, over systems of different shapes so that the shared
scratch is reused with a different layout.  Collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

import mpc_tdse
from mpc_tdse.systems import random_system

pytestmark = pytest.mark.gpu

_dp = C.POINTER(C.c_double)


def _bind():
    L = mpc_tdse.lib()
    L.mpc_rhs_noalloc.argtypes = [C.c_int, C.POINTER(C.c_int), C.c_void_p, C.c_void_p, C.c_char,
                                  C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]
    L.mpc_rhs_noalloc.restype = C.c_int
    return L


@pytest.mark.parametrize("g", ["l", "v"])
def test_noalloc_rhs_matches_context_rhs(g):
    import torch

    L = _bind()
    shapes = [[300, 513, 260, 777, 129], [5, 7, 6, 4, 9], [298] * 6]
    for k, shape in enumerate(shapes):
        s = random_system(shape, gauge=g, seed=20 + k, e_max=12.0)
        rng = np.random.default_rng(30 + k)
        x = rng.standard_normal(s.ntot) + 1j * rng.standard_normal(s.ntot)
        F = 0.37 if k % 2 == 0 else -1.1
        with mpc_tdse.Context.from_system(s) as ctx:
            want = ctx.rhs(F, x)
        dev = torch.device("cuda", 0)
        d_eig = torch.from_numpy(s.eig.copy()).to(dev)
        d_dip = torch.from_numpy(s.dip.copy()).to(dev)
        d_x = torch.from_numpy(x.view(np.float64).copy()).to(dev)
        d_out = torch.empty_like(d_x)
        n = np.ascontiguousarray(s.n, dtype=np.int32)
        stream = torch.cuda.current_stream(dev)
        scale = max(1.0, float(np.max(np.abs(want))))
        for call in range(2):
            d_out.fill_(float("nan"))
            rc = L.mpc_rhs_noalloc(len(n) - 1, n.ctypes.data_as(C.POINTER(C.c_int)),
                                   d_eig.data_ptr(), d_dip.data_ptr(), g.encode(), F,
                                   d_x.data_ptr(), d_out.data_ptr(), stream.cuda_stream)
            assert rc == 0, mpc_tdse.last_error()
            torch.cuda.synchronize()
            got = d_out.cpu().numpy().view(np.complex128)
            assert np.all(np.isfinite(got))
            assert np.max(np.abs(got - want)) <= 1e-13 * scale, (shape, call)


def test_noalloc_rejects_systems_beyond_its_scratch():
    import torch

    L = _bind()
    dev = torch.device("cuda", 0)
    buf = torch.zeros(16, dtype=torch.float64, device=dev)
    # 3 blocks of 40000 states: 2 x 157 column strips, beyond the 256 the
    # static partial-slot table holds
    n = np.array([40000, 40000, 40000], dtype=np.int32)
    rc = L.mpc_rhs_noalloc(2, n.ctypes.data_as(C.POINTER(C.c_int)), buf.data_ptr(),
                           buf.data_ptr(), b"l", 0.1, buf.data_ptr(), buf.data_ptr(), None)
    assert rc == -1
    assert "column strips" in mpc_tdse.last_error()
    # 100 strips, but 100 x 40000 row partials of 16 B = 64 MB: beyond the
    # 16 MiB static array
    n = np.array([40000, 25600], dtype=np.int32)
    rc = L.mpc_rhs_noalloc(1, n.ctypes.data_as(C.POINTER(C.c_int)), buf.data_ptr(),
                           buf.data_ptr(), b"l", 0.1, buf.data_ptr(), buf.data_ptr(), None)
    assert rc == -1
    assert "static maximum" in mpc_tdse.last_error()


def test_noalloc_refuses_misaligned_views_before_launch():
    import torch

    L = _bind()
    s = random_system([40, 50, 30], gauge="l", seed=5, e_max=8.0)
    dev = torch.device("cuda", 0)
    d_eig = torch.from_numpy(s.eig.copy()).to(dev)
    d_dip = torch.from_numpy(s.dip.copy()).to(dev)
    d_x = torch.zeros(2 * s.ntot + 2, dtype=torch.float64, device=dev)
    d_out = torch.zeros(2 * s.ntot + 2, dtype=torch.float64, device=dev)
    n = np.ascontiguousarray(s.n, dtype=np.int32)
    np_ = n.ctypes.data_as(C.POINTER(C.c_int))
    # a complex view starting one double in: 8-byte but not 16-byte aligned
    for xp, op in ((d_x.data_ptr() + 8, d_out.data_ptr()), (d_x.data_ptr(), d_out.data_ptr() + 8)):
        rc = L.mpc_rhs_noalloc(len(n) - 1, np_, d_eig.data_ptr(), d_dip.data_ptr(), b"l", 0.2,
                               xp, op, None)
        assert rc == -1
        assert "16-byte aligned" in mpc_tdse.last_error()
    rc = L.mpc_rhs_noalloc(len(n) - 1, np_, d_eig.data_ptr() + 4, d_dip.data_ptr(), b"l", 0.2,
                           d_x.data_ptr(), d_out.data_ptr(), None)
    assert rc == -1
    assert "8-byte aligned" in mpc_tdse.last_error()
    # nothing was launched: the output buffer is untouched and the device is fine
    torch.cuda.synchronize()
    assert float(d_out.abs().sum()) == 0.0
    rc = L.mpc_rhs_noalloc(len(n) - 1, np_, d_eig.data_ptr(), d_dip.data_ptr(), b"l", 0.2,
                           d_x.data_ptr(), d_out.data_ptr(), None)
    assert rc == 0, mpc_tdse.last_error()
    torch.cuda.synchronize()
