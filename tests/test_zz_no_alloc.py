"""topx_ku_noalloc: the allocation-free form of topx_ku, called through the C ABI.

topx_ku allocates temporary device buffers on each call.  Callers whose device memory belongs
to another allocator (MATLAB gpuArray, a framework's caching pool) or whose loop must not call
cudaMalloc/cudaFree use topx_ku_noalloc instead: they pass device vectors and the call takes
its scratch from a fixed 32 MiB static device array.  This file checks, on two calls in a row
and with two different models (so the second call runs on scratch that still holds the first
call's data), that its K*u equals topx_ku's within the 1e-13 relative bar of the other K*u
parity tests, and that a model too large for the fixed scratch is refused with TOPX_ERR_ARG.
The test owns its device buffers and allocates them itself, as such a caller's allocator would.
The file is named so that pytest collects it last; it also passes when run alone.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

H2D, D2H = 1, 2
KU_REL_TOL = 1e-13


def _cudart():
    for name in ("libcudart.so", "libcudart.so.12", "/usr/local/cuda/lib64/libcudart.so"):
        try:
            rt = C.CDLL(name)
        except OSError:
            continue
        rt.cudaMalloc.argtypes = [C.POINTER(C.c_void_p), C.c_size_t]
        rt.cudaFree.argtypes = [C.c_void_p]
        rt.cudaMemcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
        rt.cudaMemset.argtypes = [C.c_void_p, C.c_int, C.c_size_t]
        rt.cudaMemsetAsync.argtypes = [C.c_void_p, C.c_int, C.c_size_t, C.c_void_p]
        rt.cudaMemcpyAsync.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int, C.c_void_p]
        rt.cudaMallocHost.argtypes = [C.POINTER(C.c_void_p), C.c_size_t]
        rt.cudaFreeHost.argtypes = [C.c_void_p]
        rt.cudaDeviceSynchronize.argtypes = []
        return rt
    pytest.skip("libcudart not found")


class _DeviceVector:
    """A caller-owned FP64 device vector (allocated by the test, not by the library)."""

    def __init__(self, rt, n):
        self.rt, self.n, self.p = rt, n, C.c_void_p()
        assert rt.cudaMalloc(C.byref(self.p), 8 * n) == 0

    def upload(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        assert self.rt.cudaMemcpy(self.p, a.ctypes.data, 8 * self.n, H2D) == 0

    def poison(self):
        assert self.rt.cudaMemset(self.p, 0xFF, 8 * self.n) == 0  # all-NaN

    def download(self):
        out = np.empty(self.n)
        assert self.rt.cudaMemcpy(out.ctypes.data, self.p, 8 * self.n, D2H) == 0
        return out

    def free(self):
        self.rt.cudaFree(self.p)


def _model(vox, seed):
    from top3d_xl_b200 import Context
    ctx = Context("fp64")
    ctx.load_voxels(vox)
    rng = np.random.default_rng(seed)
    x = rng.uniform(0.05, 1.0, ctx.numElements)
    ctx.set_moduli(1e-9 + x ** 3 * (1.0 - 1e-9))  # also creates the context's device state
    return ctx


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_ku_noalloc_matches_topx_ku_on_two_calls():
    rt = _cudart()
    rng = np.random.default_rng(11)
    irregular = rng.random((13, 27, 11)) < 0.75
    irregular[:, 0, :] = True
    irregular[:, -1, :] = True
    # first a full cuboid, then a smaller irregular domain: the second call's grid has nodes
    # outside the domain whose scratch entries still hold the first call's values
    for call, (vox, seed) in enumerate([(np.ones((16, 32, 16), bool), 1), (irregular, 2)]):
        ctx = _model(vox, seed)
        ndof = ctx.numDOFs
        u = np.random.default_rng(100 + call).standard_normal(ndof)
        y_ref = ctx.ku(u)
        du, dy = _DeviceVector(rt, ndof), _DeviceVector(rt, ndof)
        try:
            du.upload(u)
            dy.poison()
            st = ctx.lib.topx_ku_noalloc(ctx._h, du.p, dy.p, ndof)
            assert st == 0, ctx.lib.topx_last_error(ctx._h)
            y = dy.download()
        finally:
            du.free()
            dy.free()
            ctx.close()
        assert np.all(np.isfinite(y))
        assert _rel(y, y_ref) <= KU_REL_TOL, (call, _rel(y, y_ref))


def test_ku_noalloc_refuses_models_beyond_the_fixed_scratch():
    rt = _cudart()
    ctx = _model(np.ones((90, 90, 90), bool), 3)  # 91^3 = 753,571 grid nodes > 699,040
    try:
        ndof = ctx.numDOFs
        du, dy = _DeviceVector(rt, ndof), _DeviceVector(rt, ndof)
        try:
            st = ctx.lib.topx_ku_noalloc(ctx._h, du.p, dy.p, ndof)
        finally:
            du.free()
            dy.free()
        assert st == -1  # TOPX_ERR_ARG
        assert b"fixed scratch" in ctx.lib.topx_last_error(ctx._h)
    finally:
        ctx.close()


def test_ku_noalloc_runs_after_work_queued_on_the_default_stream():
    """A gpuArray-style caller writes u on the legacy default stream and calls at once, with no
    synchronisation in between: the call must see the finished u (the stream 0 work is first
    a NaN fill of u, then the asynchronous copy of its values from page-locked memory)."""
    rt = _cudart()
    ctx = _model(np.ones((24, 48, 24), bool), 4)
    hbuf = C.c_void_p()
    try:
        ndof = ctx.numDOFs
        u = np.random.default_rng(7).standard_normal(ndof)
        y_ref = ctx.ku(u)
        assert rt.cudaMallocHost(C.byref(hbuf), 8 * ndof) == 0
        C.memmove(hbuf, u.ctypes.data, 8 * ndof)
        du, dy = _DeviceVector(rt, ndof), _DeviceVector(rt, ndof)
        try:
            for _ in range(2):
                assert rt.cudaMemsetAsync(du.p, 0xFF, 8 * ndof, None) == 0
                assert rt.cudaMemcpyAsync(du.p, hbuf, 8 * ndof, H2D, None) == 0
                st = ctx.lib.topx_ku_noalloc(ctx._h, du.p, dy.p, ndof)
                assert st == 0, ctx.lib.topx_last_error(ctx._h)
                y = dy.download()
                assert np.all(np.isfinite(y))
                assert _rel(y, y_ref) <= KU_REL_TOL, _rel(y, y_ref)
        finally:
            rt.cudaDeviceSynchronize()
            du.free()
            dy.free()
    finally:
        if hbuf.value:
            rt.cudaFreeHost(hbuf)
        ctx.close()
