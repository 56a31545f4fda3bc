"""The allocation-free GEMV entry point, gatlas_matvec_f32_noalloc.

Some callers cannot call cudaMalloc: code running inside a host framework
that owns (or has reserved) all of the device memory, and latency-critical
code that must not trigger the device-wide synchronisation that cudaMalloc
and cudaFree imply.  For them the library offers a GEMV that takes its
scratch (the column-major path's partial sums and arrival counters) from a
fixed 1 MiB device array inside the library instead of allocating it.

These tests call that entry point through the C ABI, on both engines (plain
loads and TMA tiles), and compare it with the regular entry point,
gatlas_matvec_f32, and with the FP64 oracle, within the GEMV tolerance used by
the other tests (normwise 4*N*u), on two calls in a row -- the second call finds
the array holding the first call's partial sums and counters and must clear
what has to start at zero.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

import gatlas_b200 as g
import oracle

pytestmark = pytest.mark.gpu
U32 = 2.0 ** -24


def _noalloc():
    fn = g.lib().gatlas_matvec_f32_noalloc
    fn.argtypes = [ctypes.POINTER(g.MatvecDesc), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return fn


@pytest.mark.parametrize("engine", ["buffer", "image"])
@pytest.mark.parametrize("trans_a", [1, 0])
@pytest.mark.parametrize("M,N", [(4096, 3000), (1024, 16384), (332, 776)])
def test_noalloc_matches_regular_entry_point(cuda, engine, trans_a, M, N):
    import torch
    fn = _noalloc()
    Ah = oracle.uniform(M * N, seed=M + N)
    xh = oracle.uniform(N, seed=N)
    A = torch.from_numpy(Ah).to(cuda)
    x = torch.from_numpy(xh).to(cuda)
    y_ref = g.matvec(A, x, M, N, trans_a=trans_a, engine=engine)   # regular entry point
    d = g.matvec_desc(M, N, trans_a=trans_a, engine=engine)
    outs = []
    for _ in range(2):                                      # two calls in a row
        y = torch.full((M,), float("nan"), device=cuda)
        rc = fn(ctypes.byref(d), g._ptr(A), g._ptr(x), g._ptr(y), g._stream())
        assert rc == 0, g.last_error()
        torch.cuda.synchronize()
        outs.append(y.cpu().numpy())
    assert g.device_faults() == 0
    ref = y_ref.cpu().numpy()
    exact = oracle.matvec(Ah, xh, M, N, trans_a, mode=oracle.F64)
    for y in outs:
        assert np.all(np.isfinite(y))
        assert oracle.normwise_error(y, ref) <= 4 * N * U32
        assert oracle.normwise_error(y, exact) <= 4 * N * U32


@pytest.mark.parametrize("engine", ["buffer", "image"])
def test_noalloc_general_form_two_calls(cuda, engine):
    # y = alpha*A^T x + beta*y, and a different problem on the second call
    import torch
    fn = _noalloc()
    for M, N, seed in ((2048, 5000, 1), (640, 20000, 2)):
        Ah, xh, yh = oracle.uniform(M * N, seed=seed), oracle.uniform(N, seed=seed + 10), oracle.uniform(M, seed=seed + 20)
        A, x, y0 = (torch.from_numpy(t).to(cuda) for t in (Ah, xh, yh))
        y_ref = g.matvec(A, x, M, N, y=y0.clone(), trans_a=True, gemv=True, alpha=0.5, beta=-1.5, engine=engine)
        y = y0.clone()
        d = g.matvec_desc(M, N, trans_a=True, gemv=True, alpha=0.5, beta=-1.5, engine=engine)
        assert fn(ctypes.byref(d), g._ptr(A), g._ptr(x), g._ptr(y), g._stream()) == 0, g.last_error()
        torch.cuda.synchronize()
        assert g.device_faults() == 0
        got = y.cpu().numpy()
        assert oracle.normwise_error(got, y_ref.cpu().numpy()) <= 4 * N * U32
        exact = oracle.matvec(Ah, xh, M, N, 1, mode=oracle.F64, gemv=1, cin=yh, alpha=0.5, beta=-1.5)
        assert oracle.normwise_error(got, exact) <= 4 * N * U32


def test_noalloc_rejects_null_descriptor():
    fn = _noalloc()
    assert fn(None, None, None, None, None) == g.ERR_INVALID
    assert "null descriptor" in g.last_error()
