"""The allocation-free GEMV entry point, gatlas_matvec_f32_noalloc.

Some callers cannot call cudaMalloc: code running inside a host framework
that owns (or has reserved) all of the device memory, and latency-critical
code that must not trigger the device-wide synchronisation that cudaMalloc
and cudaFree imply.  For them the library offers a GEMV that takes its
scratch (the column-major path's partial sums and arrival counters) from a
fixed 1 MiB device array inside the library instead of allocating it.

These tests call that entry point through the C ABI and compare it with the
regular entry point, gatlas_matvec_f32, within the GEMV tolerance used by the
other tests (normwise 4*N*u), on two calls in a row -- the second call finds
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


@pytest.mark.parametrize("trans_a", [1, 0])
@pytest.mark.parametrize("M,N", [(4096, 3000), (1024, 16384), (333, 777)])
def test_noalloc_matches_regular_entry_point(cuda, trans_a, M, N):
    import torch
    fn = _noalloc()
    A = torch.from_numpy(oracle.uniform(M * N, seed=M + N)).to(cuda)
    x = torch.from_numpy(oracle.uniform(N, seed=N)).to(cuda)
    y_ref = g.matvec(A, x, M, N, trans_a=trans_a)          # regular entry point
    d = g.matvec_desc(M, N, trans_a=trans_a)
    outs = []
    for _ in range(2):                                      # two calls in a row
        y = torch.full((M,), float("nan"), device=cuda)
        rc = fn(ctypes.byref(d), g._ptr(A), g._ptr(x), g._ptr(y), g._stream())
        assert rc == 0, g.last_error()
        torch.cuda.synchronize()
        outs.append(y.cpu().numpy())
    ref = y_ref.cpu().numpy()
    for y in outs:
        assert np.all(np.isfinite(y))
        assert oracle.normwise_error(y, ref) <= 4 * N * U32


def test_noalloc_general_form_two_calls(cuda):
    # y = alpha*A^T x + beta*y, and a different problem on the second call
    import torch
    fn = _noalloc()
    for M, N, seed in ((2048, 5000, 1), (640, 20000, 2)):
        A = torch.from_numpy(oracle.uniform(M * N, seed=seed)).to(cuda)
        x = torch.from_numpy(oracle.uniform(N, seed=seed + 10)).to(cuda)
        y0 = torch.from_numpy(oracle.uniform(M, seed=seed + 20)).to(cuda)
        y_ref = g.matvec(A, x, M, N, y=y0.clone(), trans_a=True, gemv=True, alpha=0.5, beta=-1.5)
        y = y0.clone()
        d = g.matvec_desc(M, N, trans_a=True, gemv=True, alpha=0.5, beta=-1.5)
        assert fn(ctypes.byref(d), g._ptr(A), g._ptr(x), g._ptr(y), g._stream()) == 0, g.last_error()
        torch.cuda.synchronize()
        assert oracle.normwise_error(y.cpu().numpy(), y_ref.cpu().numpy()) <= 4 * N * U32


def test_noalloc_rejects_null_descriptor():
    fn = _noalloc()
    assert fn(None, None, None, None, None) == g.ERR_INVALID
    assert "null descriptor" in g.last_error()
