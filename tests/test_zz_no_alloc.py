"""The allocation-free residual norm, cosa_gpu_resg_rms_noalloc.

Some callers cannot allocate device memory: a Fortran driver whose device
arrays are owned and pooled by another runtime, or code running where a new
cudaMalloc would fail or is not allowed.  For them the library offers the
residual RMS with its scratch in a fixed static device array instead of
context-owned buffers.  This test calls it through the C-ABI twice in a row
(different residuals, with and without the multigrid forcing term) and
checks each result against the context-based cosa_gpu_resg_rms, within the
tolerance the other residual-norm checks use (1e-9 relative); with k-omega
(npde = 7) and harmonic balance (every snapshot enters the norm, as in
resg_rms_hb) it checks against the same norm computed in numpy.

The file name sorts last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from cosa_b200 import cases, gpu

import casekit

pytestmark = pytest.mark.gpu
RTOL = 1e-9


def _noalloc(lib, tables, npde, nharms, res, rhs, out, stream):
    # the result is read back on `stream`, so the call must be issued on it too
    dims = np.ascontiguousarray(tables.dims.ravel(), dtype=np.int32)
    st = lib.cosa_gpu_resg_rms_noalloc(
        C.c_int32(tables.nblocks), dims.ctypes.data_as(C.POINTER(C.c_int32)), C.c_int32(npde),
        C.c_int32(nharms), C.c_void_p(res.ptr), C.c_void_p(rhs.ptr if rhs is not None else None),
        C.c_void_p(out.ptr), C.c_void_p(stream))
    assert st == 0, st
    return out.download()


def test_noalloc_rms_matches_context_rms():
    case = casekit.small_partitioned()
    p = case.params
    lib = gpu.load()
    ctx = gpu.Context([case.tables], p)
    rng = np.random.default_rng(42)
    n = ctx.alloc_p3().n
    res = ctx.alloc_p3()
    rhs = ctx.alloc_p3()
    out = gpu.DevArray(ctx, p.npde + 1)
    for call, with_rhs in enumerate((False, True)):
        res.upload(rng.standard_normal(n) * 10.0 ** -(3 + call))
        rhs.upload(rng.standard_normal(n) * 1e-4)
        want = ctx.resg_rms(1, res, rhs if with_rhs else None)
        got = _noalloc(lib, case.tables, p.npde, p.nharms, res, rhs if with_rhs else None, out, ctx.stream())
        np.testing.assert_allclose(got, want, rtol=RTOL, atol=0)
    ctx.close()


def _numpy_rms(tables, flat, npde, nsnap, rhs=None):
    """resg_rms / resg_rms_hb (src/cosa.f90:4458-4697) in numpy: squares of
    every interior cell of every snapshot, over ncell * nsnap."""
    d = flat if rhs is None else flat - rhs
    sums = np.zeros(npde)
    ncell = 0
    for v in cases.p3_views(tables, d, npde, nsnap):
        iv = cases.interior(v)
        sums += (iv ** 2).sum(axis=(0, 1, 2, 4))
        ncell += iv.shape[0] * iv.shape[1] * iv.shape[2]
    out = np.sqrt(sums / (ncell * nsnap))
    return np.append(out, np.sqrt(sums.sum() / (ncell * nsnap) / npde))


@pytest.mark.parametrize("npde,nharms", [(7, 0), (5, 1), (7, 1)])
def test_noalloc_rms_harmonic_balance_and_turbulence(npde, nharms):
    # harmonic balance: every snapshot enters, divided by ncell * (2 nharms + 1)
    case = casekit.small_partitioned()
    lib = gpu.load()
    ctx = gpu.Context([case.tables], case.params)
    S = 2 * nharms + 1
    n = sum((im + 3) * (jm + 3) * (km + 3) for im, jm, km in case.tables.dims) * npde * S
    rng = np.random.default_rng(7 + npde + nharms)
    res, rhs = gpu.DevArray(ctx, n), gpu.DevArray(ctx, n)
    out = gpu.DevArray(ctx, npde + 1)
    for call in range(2):
        r = rng.standard_normal(n) * 10.0 ** -(2 + call)
        h = rng.standard_normal(n) * 1e-4 if call else None
        res.upload(r)
        if h is not None:
            rhs.upload(h)
        got = _noalloc(lib, case.tables, npde, nharms, res, rhs if h is not None else None, out, ctx.stream())
        np.testing.assert_allclose(got, _numpy_rms(case.tables, r, npde, S, h), rtol=RTOL, atol=0)
    ctx.close()


def test_noalloc_rms_rejects_oversized_block_table():
    lib = gpu.load()
    dims = np.full(3 * 5000, 9, dtype=np.int32)
    st = lib.cosa_gpu_resg_rms_noalloc(C.c_int32(5000), dims.ctypes.data_as(C.POINTER(C.c_int32)), C.c_int32(5),
                                       C.c_int32(0), C.c_void_p(None), C.c_void_p(None), C.c_void_p(None),
                                       C.c_void_p(None))
    assert st == 0x10  # COSA_ERR_ARG, before any device work
