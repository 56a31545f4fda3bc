"""Operands past 2^31 elements: every engine addresses its buffers with 64-bit
element offsets.  The inputs are generated on the device by the seeded
counter-based fill, so the oracle regenerates any window of them by offset
and checks the results there (the window that straddles element 2^31 and the
last rows), without holding the full operands on the host.

Sizes: SAXPY 2^31 + 4099 elements per vector; GEMV 65539 x 32784 (2.15 G
elements of A); GEMM C of 46400 x 46400 (2.15 G elements), one instance or
the last of a batch of three.  Each test holds 9-18 GB on the device."""
import numpy as np
import pytest

import gatlas_b200 as g
import oracle

pytestmark = pytest.mark.gpu
U32 = 2.0 ** -24
TWO31 = 1 << 31
# sign*2^e operands: every product is exact in every engine, only the
# accumulation rounds (FP8: inside each 128-deep block, then FP32 promotion)
PIPE_TOL = 2.0 ** -12


def _free():
    import torch
    torch.cuda.synchronize()
    torch.cuda.empty_cache()


@pytest.mark.parametrize("engine", ["buffer", "image"])
def test_saxpy_past_2_31(cuda, engine):
    import torch
    n = TWO31 + 4099
    x = torch.empty(n, dtype=torch.float32, device=cuda)
    y = torch.empty(n, dtype=torch.float32, device=cuda)
    g.fill(x, "uniform", seed=11)
    g.fill(y, "uniform", seed=12)
    g.saxpy(0.75, x, y, out=y, engine=engine)
    torch.cuda.synchronize()
    assert g.device_faults() == 0
    for lo, hi in ((0, 4096), (TWO31 - 3000, TWO31 + 3000), (n - 8192, n)):
        got = y[lo:hi].cpu().numpy()
        ref = oracle.saxpy(0.75, oracle.uniform(hi - lo, 11, offset=lo), oracle.uniform(hi - lo, 12, offset=lo),
                           mode=oracle.FMA)
        assert np.array_equal(got, ref), (lo, hi)
    del x, y
    _free()


@pytest.mark.parametrize("ta", [0, 1])
def test_matvec_past_2_31(cuda, ta):
    import torch
    M, N = 65539, 32784
    assert M * N > TWO31
    A = torch.empty(M * N, dtype=torch.float32, device=cuda)
    x = torch.empty(N, dtype=torch.float32, device=cuda)
    g.fill(A, "uniform", seed=21)
    g.fill(x, "uniform", seed=22)
    y = g.matvec(A, x, M, N, trans_a=ta)
    torch.cuda.synchronize()
    assert g.device_faults() == 0
    hx = oracle.uniform(N, 22)
    if ta == 0:
        # row-major M x N: rows 65503.. straddle element 2^31
        windows = [(TWO31 // N - 8, TWO31 // N + 8), (M - 40, M)]
    else:
        # stored N x M (element (i, j) at j*M + i): every y[i] reads past 2^31
        windows = [(0, 16), (M - 24, M)]
    for lo, hi in windows:
        w = hi - lo
        if ta == 0:
            Aw = oracle.uniform(w * N, 21, offset=lo * N)
        else:
            Aw = np.concatenate([oracle.uniform(w, 21, offset=j * M + lo) for j in range(N)])
        ref = oracle.matvec(Aw, hx, w, N, ta, mode=oracle.F64)
        got = y[lo:hi].cpu().numpy()
        assert oracle.normwise_error(got, ref) <= 4 * N * U32, (lo, hi)
    del A, x, y
    _free()


ENGINES = ["tc_bf16", "tc_split3", "tc_split6", "tc_fp8", "buffer", "image"]


def _tol(engine, K):
    return PIPE_TOL if engine == "tc_fp8" else 4 * K * U32


def _check_rows(C, lo, hi, M, N, K, engine, seed_a, seed_b, instance=0, dtype=np.float32):
    w = hi - lo
    base_a = instance * M * K
    if dtype == np.float32:
        Aw = oracle.pow2(w * K, seed_a, offset=base_a + lo * K)
        B = oracle.pow2(K * N, seed_b, offset=instance * K * N)
    else:
        Aw = oracle.uniform(w * K, seed_a, offset=base_a + lo * K, dtype=np.float64)
        B = oracle.uniform(K * N, seed_b, offset=instance * K * N, dtype=np.float64)
    got = C[instance * M * N + lo * N:instance * M * N + hi * N].cpu().numpy()
    if dtype == np.float64:
        # DGEMM accumulates each element by sequential FMAs over k: bit-exact
        ref = oracle.matmul(Aw, B, w, N, K, mode=oracle.FMA, dtype=np.float64)
        assert np.array_equal(got, ref), (engine, lo, hi)
        return
    ref = oracle.matmul(Aw, B, w, N, K, mode=oracle.F64)
    assert oracle.normwise_error(got, ref) <= _tol(engine, K), (engine, lo, hi)


@pytest.mark.parametrize("engine", ENGINES)
def test_matmul_c_past_2_31(cuda, engine):
    import torch
    M = N = 46400
    K = 64
    assert M * N > TWO31
    A = torch.empty(M * K, dtype=torch.float32, device=cuda)
    B = torch.empty(K * N, dtype=torch.float32, device=cuda)
    g.fill(A, "pow2", seed=31)
    g.fill(B, "pow2", seed=32)
    C = torch.full((M * N,), float("nan"), dtype=torch.float32, device=cuda)
    g.matmul(A, B, M, N, K, C=C, engine=engine)
    torch.cuda.synchronize()
    assert g.device_faults() == 0
    # 46208 is a 128-row block boundary; row 46282 holds element 2^31
    _check_rows(C, 46208, 46336, M, N, K, engine, 31, 32)
    _check_rows(C, 46336, M, M, N, K, engine, 31, 32)
    _check_rows(C, 0, 8, M, N, K, engine, 31, 32)
    del A, B, C
    _free()


@pytest.mark.parametrize("engine", ["tc_split3", "tc_fp8", "buffer"])
def test_batched_matmul_past_2_31(cuda, engine):
    import torch
    M = N = 26880
    K, P = 32, 3
    assert P * M * N > TWO31
    A = torch.empty(P * M * K, dtype=torch.float32, device=cuda)
    B = torch.empty(P * K * N, dtype=torch.float32, device=cuda)
    g.fill(A, "pow2", seed=41)
    g.fill(B, "pow2", seed=42)
    C = torch.full((P * M * N,), float("nan"), dtype=torch.float32, device=cuda)
    g.matmul(A, B, M, N, K, C=C, engine=engine, batch=P)
    torch.cuda.synchronize()
    assert g.device_faults() == 0
    # instance 2 starts at element 2 * M * N = 1.45 G and ends past 2^31
    _check_rows(C, M - 136, M, M, N, K, engine, 41, 42, instance=2)
    _check_rows(C, 0, 8, M, N, K, engine, 41, 42, instance=1)
    del A, B, C
    _free()


def test_dgemm_c_past_2_31(cuda):
    import torch
    M = N = 46400
    K = 16
    A = torch.empty(M * K, dtype=torch.float64, device=cuda)
    B = torch.empty(K * N, dtype=torch.float64, device=cuda)
    g.fill(A, "uniform", seed=51)
    g.fill(B, "uniform", seed=52)
    C = torch.full((M * N,), float("nan"), dtype=torch.float64, device=cuda)
    g.matmul(A, B, M, N, K, C=C, engine="buffer")
    torch.cuda.synchronize()
    assert g.device_faults() == 0
    _check_rows(C, 46272, M, M, N, K, "buffer", 51, 52, dtype=np.float64)
    del A, B, C
    _free()


def test_grouped_instance_past_2_31(cuda):
    import torch
    M = N = 46400
    K = 64
    A = torch.empty(M * K, dtype=torch.float32, device=cuda)
    B = torch.empty(K * N, dtype=torch.float32, device=cuda)
    g.fill(A, "pow2", seed=31)
    g.fill(B, "pow2", seed=32)
    C = torch.full((M * N,), float("nan"), dtype=torch.float32, device=cuda)
    sa, sb = oracle.uniform(200 * 96, 61), oracle.uniform(96 * 300, 62)
    small = dict(A=torch.from_numpy(sa).to(cuda), B=torch.from_numpy(sb).to(cuda),
                 C=torch.zeros(200 * 300, dtype=torch.float32, device=cuda), m=200, n=300, k=96)
    inst = [dict(A=A, B=B, C=C, m=M, n=N, k=K), small]
    g.Grouped(inst, engine="tc_split3").prepare().run()
    torch.cuda.synchronize()
    assert g.device_faults() == 0
    _check_rows(C, 46208, M, M, N, K, "tc_split3", 31, 32)
    ref = oracle.matmul(sa, sb, 200, 300, 96, mode=oracle.F64)
    assert oracle.normwise_error(small["C"].cpu().numpy(), ref) <= 8e-6
    del A, B, C, inst, small
    _free()
