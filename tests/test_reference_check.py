"""The paranoid check's device reference in both arithmetics, bit for bit
against the oracle's restatement of the same loops:

- fused=False: the reference's host check loops, every product and sum
  rounded separately (KernelMatmulBuffer.hpp:124-143,
  KernelMatvecBuffer.hpp:122-138, KernelSaxpyBuffer.hpp:118-120) -- the
  oracle's REFHOST mode;
- fused=True: the generated kernels' mad chain (KernelMatmulBuffer.hpp:302-337)
  -- the oracle's FMA mode.

Then the plugin's paranoid check in the reference's arithmetic: its absdiff
equals the oracle's absdiff between the engine's result and REFHOST."""
import numpy as np
import pytest

import gatlas_b200 as g
import oracle
from gatlas_b200.plugin import Kernel

pytestmark = pytest.mark.gpu
MODES = {False: oracle.REFHOST, True: oracle.FMA}


def _t(cuda, a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("fused", [False, True])
@pytest.mark.parametrize("ta,tb", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_matmul_reference_bit_exact(cuda, dtype, fused, ta, tb):
    M, N, K, P = 130, 97, 301, 2
    A = oracle.uniform(P * M * K, seed=1 + ta, dtype=dtype)
    B = oracle.uniform(P * K * N, seed=2 + tb, dtype=dtype)
    C0 = oracle.uniform(P * M * N, seed=3, dtype=dtype)
    for gemm, alpha, beta in ((0, 1.0, 0.0), (1, 0.75, -1.25), (1, 2.0, 0.0)):
        got = g.reference_matmul(_t(cuda, A), _t(cuda, B), M, N, K, fused=fused, Cin=_t(cuda, C0), trans_a=ta,
                                 trans_b=tb, gemm=gemm, alpha=alpha, beta=beta, batch=P).cpu().numpy()
        want = oracle.matmul(A, B, M, N, K, ta, tb, mode=MODES[fused], gemm=gemm, Cin=C0, alpha=alpha, beta=beta,
                             packed=P, dtype=dtype)
        assert np.array_equal(got, want), (gemm, alpha, beta)


def test_the_two_arithmetics_differ(cuda):
    # on drand48-style positive inputs the separately rounded chain and the
    # fused chain part in the last bits: the modes are really distinct
    M = N = K = 256
    A = oracle.fillrand(M * K)
    B = oracle.fillrand(K * N)
    f = g.reference_matmul(_t(cuda, A), _t(cuda, B), M, N, K, fused=True).cpu().numpy()
    u = g.reference_matmul(_t(cuda, A), _t(cuda, B), M, N, K, fused=False).cpu().numpy()
    assert not np.array_equal(f, u)
    assert np.array_equal(u, oracle.matmul(A, B, M, N, K, mode=oracle.REFHOST))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("fused", [False, True])
@pytest.mark.parametrize("ta", [0, 1])
def test_matvec_reference_bit_exact(cuda, dtype, fused, ta):
    M, N, P = 1000, 777, 3
    A = oracle.uniform(P * M * N, seed=5 + ta, dtype=dtype)
    x = oracle.uniform(P * N, seed=6, dtype=dtype)
    y0 = oracle.uniform(P * M, seed=7, dtype=dtype)
    for gemv, alpha, beta in ((0, 1.0, 0.0), (1, -0.5, 1.5)):
        got = g.reference_matvec(_t(cuda, A), _t(cuda, x), M, N, fused=fused, yin=_t(cuda, y0), trans_a=ta,
                                 gemv=gemv, alpha=alpha, beta=beta, batch=P).cpu().numpy()
        want = oracle.matvec(A, x, M, N, ta, mode=MODES[fused], gemv=gemv, cin=y0, alpha=alpha, beta=beta,
                             packed=P, dtype=dtype)
        assert np.array_equal(got, want)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("fused", [False, True])
def test_saxpy_reference_bit_exact(cuda, dtype, fused):
    n = 1_000_003
    x = oracle.uniform(n, seed=8, dtype=dtype)
    y = oracle.uniform(n, seed=9, dtype=dtype)
    got = g.reference_saxpy(0.3, _t(cuda, x), _t(cuda, y), fused=fused).cpu().numpy()
    assert np.array_equal(got, oracle.saxpy(0.3, x, y, mode=MODES[fused], dtype=dtype))


def test_reference_rejects_strided_layouts(cuda):
    import torch
    A = torch.zeros(64, device=cuda)
    with pytest.raises(g.GatlasError, match="dense"):
        d = g.matmul_desc(4, 4, 4, lda=8)
        import ctypes
        g.check(g.lib().gatlas_reference_matmul(0, 1, ctypes.byref(d), g._ptr(A), g._ptr(A), None, g._ptr(A),
                                                g._stream()))


@pytest.mark.parametrize("fused", [True, False])
def test_plugin_paranoid_check_in_either_arithmetic(cuda, fused):
    # Random drand48 inputs (KernelMatmulBuffer.hpp:104-116).  Against the
    # fused reference the SIMT engine matches bit for bit: absdiff 0.  Against
    # the reference's own separately rounded host loop the fmaf chain differs
    # in the last bits of most elements, and the reference's pass rule
    # (absdiff < 1/length, OCLAppUtil.hpp:212-264) decides on that absdiff.
    M = N = K = 128
    k = Kernel("matmul", "float4")
    k.paranoid_check(fused=fused)
    usec = k.bench_run([1, 0, M, N, K, 0, 0, 16, 16, 8, 4, 0])
    diff = k.last_check()
    if fused:
        assert diff == 0.0 and usec > 0
    else:
        assert diff > 0.0
        assert (usec > 0) == (diff < 1.0 / (M * N))
