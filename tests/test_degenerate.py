"""Zero-sized problems through every compute entry point: each call returns
success, launches nothing that could touch memory, and leaves its outputs as
they were.  The reference's kernels take these sizes as empty loops
(KernelSaxpyBuffer.hpp:186-190, KernelMatvecBuffer.hpp:270-305,
KernelMatmulBuffer.hpp:259-337); the library returns before any launch.
Operand buffers hold one element so that no pointer is null."""
import numpy as np
import pytest

import gatlas_b200 as g

pytestmark = pytest.mark.gpu


def _sentinel(cuda, n):
    import torch
    return torch.full((n,), 7.0, device=cuda)


@pytest.mark.parametrize("engine", ["buffer", "image"])
def test_saxpy_n_zero(cuda, engine):
    import torch
    x = torch.ones(1, device=cuda)
    y = torch.ones(1, device=cuda)
    out = _sentinel(cuda, 1)
    rc = g.lib().gatlas_saxpy_f32(g._engine(engine), 0, 0.5, g._ptr(x), g._ptr(y), g._ptr(out), g._stream())
    assert rc == 0, g.last_error()
    torch.cuda.synchronize()
    assert out.item() == 7.0
    assert g.device_faults() == 0


@pytest.mark.parametrize("engine", ["buffer", "image"])
@pytest.mark.parametrize("ta", [0, 1])
def test_matvec_m_zero(cuda, engine, ta):
    import ctypes
    import torch
    A = torch.ones(1, device=cuda)
    x = torch.ones(1, device=cuda)
    y = _sentinel(cuda, 1)
    d = g.matvec_desc(0, 64, trans_a=ta, engine=engine)
    rc = g.lib().gatlas_matvec_f32(ctypes.byref(d), g._ptr(A), g._ptr(x), g._ptr(y), None, 0, g._stream())
    assert rc == 0, g.last_error()
    torch.cuda.synchronize()
    assert y.item() == 7.0
    assert g.device_faults() == 0


@pytest.mark.parametrize("engine", ["buffer", "image", "tc_bf16", "tc_split3", "tc_split6", "tc_fp8"])
@pytest.mark.parametrize("M,N,K", [(0, 64, 64), (64, 0, 64)])
def test_matmul_empty_output(cuda, engine, M, N, K):
    import ctypes
    import torch
    A = torch.ones(1, device=cuda)
    B = torch.ones(1, device=cuda)
    C = _sentinel(cuda, 1)
    d = g.matmul_desc(M, N, K, engine=engine)
    rc = g.lib().gatlas_matmul_f32(ctypes.byref(d), g._ptr(A), g._ptr(B), g._ptr(C), None, 0, g._stream())
    assert rc == 0, g.last_error()
    torch.cuda.synchronize()
    assert C.item() == 7.0
    assert g.device_faults() == 0


@pytest.mark.parametrize("engine", ["buffer", "tc_split3"])
def test_host_buffer_matmul_empty_output(cuda, engine):
    import ctypes
    A = np.ones(1, np.float32)
    B = np.ones(1, np.float32)
    C = np.full(1, 7.0, np.float32)
    d = g.matmul_desc(0, 64, 64, engine=engine)
    rc = g.lib().gatlas_matmul_f32_host(ctypes.byref(d), A.ctypes.data, B.ctypes.data, C.ctypes.data, None)
    assert rc == 0, g.last_error()
    assert C[0] == 7.0
    assert g.device_faults() == 0
