"""FP8 E4M3 tensor-core engine with one power-of-two FP32 scale per 128 x 128
block of each operand.  The quantisation pass is bit-exact against the
oracle's restatement (codes and scales, every layout); the contraction is
checked against the FP64 product of the dequantised operands, and its error
against the FP64 product of the original operands is reported within the
E4M3 budget."""
import numpy as np
import pytest

import gatlas_b200 as g
import oracle

pytestmark = pytest.mark.gpu
U32 = 2.0 ** -24
# contraction of the dequantised operands: FP32 accumulation inside each
# 128-deep block, promoted into FP32 registers between blocks
PIPE_TOL = 2.0 ** -12
# E4M3 keeps 3 mantissa bits (unit roundoff 2^-4) per operand
FP8_BUDGET = 2.0 ** -4


def _gpu(cuda, a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


def _rup(x, a):
    return (x + a - 1) // a * a


def _ws_views(ws, M, N, K, batch):
    """Splits a prepared FP8 workspace: [A codes][B codes][A scales][B scales]."""
    Kp = oracle.fp8_kp(K)
    mb, nb, kb = -(-M // 128), -(-N // 128), -(-K // 128)
    a_bytes, b_bytes = _rup(batch * M * Kp, 1024), _rup(batch * N * Kp, 1024)
    sa_bytes = _rup(batch * mb * kb * 4, 1024)
    h = ws.cpu().numpy()
    qa = h[:batch * M * Kp].reshape(batch, M, Kp)
    qb = h[a_bytes:a_bytes + batch * N * Kp].reshape(batch, N, Kp)
    o = a_bytes + b_bytes
    sa = h[o:o + batch * mb * kb * 4].view(np.float32).reshape(batch, mb, kb)
    sb = h[o + sa_bytes:o + sa_bytes + batch * nb * kb * 4].view(np.float32).reshape(batch, nb, kb)
    return qa, qb, sa, sb


def _oracle_quant(A, B, M, N, K, ta, tb, batch):
    qa, sa = oracle.quant_fp8(A, M, K, ta, batch=batch, src_stride=M * K)
    # B is K x N logically: K-major rows of B^T are stored directly only when tb
    qb, sb = oracle.quant_fp8(B, N, K, 0 if tb else 1, batch=batch, src_stride=K * N)
    return qa, qb, sa, sb


def _prepare(cuda, A, B, M, N, K, ta, tb, batch):
    import torch
    ws = torch.zeros(g.matmul_workspace_size(M, N, K, "tc_fp8", ta, tb, batch), dtype=torch.uint8, device=cuda)
    g.matmul_tc_prepare(_gpu(cuda, A), _gpu(cuda, B), M, N, K, ws, ta, tb, engine="tc_fp8", batch=batch)
    torch.cuda.synchronize()
    return ws


def _operands(M, N, K, batch, seed, dist="uniform"):
    if dist == "uniform":
        A = oracle.uniform(batch * M * K, seed=seed) * np.float32(3.0)
        B = oracle.uniform(batch * K * N, seed=seed + 1) * np.float32(0.01)
    else:
        A = oracle.pow2(batch * M * K, seed=seed)
        B = oracle.pow2(batch * K * N, seed=seed + 1)
    return A, B


SHAPES = [(128, 256, 128), (200, 300, 100), (257, 129, 520), (1, 1, 1), (64, 1000, 16), (384, 256, 1024)]


@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("M,N,K", SHAPES)
def test_quantisation_bit_exact(cuda, ta, tb, M, N, K):
    A, B = _operands(M, N, K, 1, seed=M + K)
    A[: min(A.size, 300)] = 0.0
    ws = _prepare(cuda, A, B, M, N, K, ta, tb, 1)
    got = _ws_views(ws, M, N, K, 1)
    want = _oracle_quant(A, B, M, N, K, ta, tb, 1)
    for x, y in zip(got, want):
        assert np.array_equal(x, y)


def test_quantisation_batch_zero_block_and_wide_range(cuda):
    M, N, K, P = 256, 256, 384, 2
    A, B = _operands(M, N, K, P, seed=4)
    A[:M * K][: 128 * K] = 0.0                                   # an all-zero scale block row
    A[M * K:] *= np.float32(2.0 ** 100)                          # second instance far from 1
    B[::7] *= np.float32(2.0 ** -30)                             # values flushed to subnormal codes / zero
    ws = _prepare(cuda, A, B, M, N, K, 0, 0, P)
    for x, y in zip(_ws_views(ws, M, N, K, P), _oracle_quant(A, B, M, N, K, 0, 0, P)):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("M,N,K", SHAPES)
def test_contraction_matches_dequantised_product(cuda, ta, tb, M, N, K):
    import torch
    A, B = _operands(M, N, K, 1, seed=2 * M + N)
    ws = _prepare(cuda, A, B, M, N, K, ta, tb, 1)
    qa, qb, sa, sb = _ws_views(ws, M, N, K, 1)
    C = torch.full((M * N,), float("nan"), device=cuda)
    g.matmul_tc_run(ws, M, N, K, C, ta, tb, engine="tc_fp8")
    torch.cuda.synchronize()
    assert g.device_faults() == 0
    ref = oracle.matmul_fp8_dequant(qa, sa, qb, sb, M, N, K)
    assert oracle.normwise_error(C.cpu().numpy(), ref) <= PIPE_TOL


def test_gemm_alpha_beta_batch(cuda):
    M, N, K, P = 160, 272, 300, 3
    A, B = _operands(M, N, K, P, seed=7)
    Cin = oracle.uniform(P * M * N, seed=9)
    C = g.matmul(_gpu(cuda, A), _gpu(cuda, B), M, N, K, C=_gpu(cuda, Cin), gemm=True, alpha=0.5, beta=-2.0,
                 engine="tc_fp8", batch=P)
    qa, qb, sa, sb = _oracle_quant(A, B, M, N, K, 0, 0, P)
    ref = oracle.matmul_fp8_dequant(qa, sa, qb, sb, M, N, K, batch=P, gemm=1, alpha=0.5, beta=-2.0, Cin=Cin)
    assert oracle.normwise_error(C.cpu().numpy(), ref) <= PIPE_TOL


def test_known_answer_c_equals_k(cuda):
    # ones: scale 2^-8, code 256, every partial and scale product exact
    M = N = K = 1024
    C = g.matmul(_gpu(cuda, np.ones(M * K, np.float32)), _gpu(cuda, np.ones(K * N, np.float32)), M, N, K,
                 engine="tc_fp8")
    assert oracle.check_pattern(C.cpu().numpy(), float(K))


@pytest.mark.parametrize("dist", ["uniform", "pow2"])
def test_error_against_fp64_of_the_original_operands(cuda, dist):
    M, N, K = 512, 512, 1024
    A, B = _operands(M, N, K, 1, seed=11, dist=dist)
    C = g.matmul(_gpu(cuda, A), _gpu(cuda, B), M, N, K, engine="tc_fp8").cpu().numpy()
    err = oracle.normwise_error(C, oracle.matmul(A, B, M, N, K, mode=oracle.F64))
    if dist == "uniform":
        assert err <= FP8_BUDGET
    else:
        # sign*2^e operands quantise exactly: only the accumulation rounds
        assert err <= PIPE_TOL


def test_full_size_error_on_the_device(cuda):
    # 4096^3 through the FP64 residual on the GPU
    import torch
    M = N = K = 4096
    A = torch.empty(M * K, device=cuda)
    B = torch.empty(K * N, device=cuda)
    g.fill(A, "uniform", seed=1)
    g.fill(B, "uniform", seed=2)
    C = g.matmul(A, B, M, N, K, engine="tc_fp8")
    fro, ref, _, _ = g.residual(A, B, C, M, N, K)
    assert fro / ref <= FP8_BUDGET
    assert g.device_faults() == 0


@pytest.mark.parametrize("extra", [1, 2, 4])
def test_segments_follow_changing_block_scales(cuda, extra):
    # scale products change along K (A's column blocks and B's row blocks are
    # scaled by different powers of two), so runs of equal scale break at the
    # changes; every promotion interval gives the dequantised product
    import torch
    M, N, K = 256, 384, 1280
    A, B = _operands(M, N, K, 1, seed=21)
    A2 = A.reshape(M, K).copy()
    B2 = B.reshape(K, N).copy()
    for kb in range(K // 128):
        A2[:, kb * 128:(kb + 1) * 128] *= np.float32(2.0 ** (kb % 3 - 1))
        B2[kb * 128:(kb + 1) * 128, :128] *= np.float32(2.0 ** (kb // 4))
    A2, B2 = A2.ravel(), B2.ravel()
    ws = _prepare(cuda, A2, B2, M, N, K, 0, 0, 1)
    qa, qb, sa, sb = _ws_views(ws, M, N, K, 1)
    assert len(set(sa[0, 0].tolist())) == 3 and len(set(sb[0, 0].tolist())) > 1
    C = torch.full((M * N,), float("nan"), device=cuda)
    g.matmul_tc_run(ws, M, N, K, C, engine="tc_fp8", extra=extra)
    torch.cuda.synchronize()
    assert g.device_faults() == 0
    ref = oracle.matmul_fp8_dequant(qa, sa, qb, sb, M, N, K)
    assert oracle.normwise_error(C.cpu().numpy(), ref) <= PIPE_TOL


def test_k_limit_of_the_fp8_engine(cuda):
    import torch
    M = N = 16
    K = 1024 * 128 + 16
    A = torch.zeros(M * K, device=cuda)
    B = torch.zeros(K * N, device=cuda)
    with pytest.raises(g.GatlasError, match="K <="):
        g.matmul(A, B, M, N, K, engine="tc_fp8")


def test_tiles_with_different_segment_plans_in_one_launch(cuda):
    # every 128-row block of A and every 128-column block of B gets its own
    # pattern of scales along K, and the instances differ too, so the tiles of
    # one launch have different numbers of segments; 180 tiles of 128 x 256 put
    # two tiles on some CTAs of the persistent kernel
    import torch
    M, N, K, P = 2304, 1280, 768, 2
    A, B = _operands(M, N, K, P, seed=41)
    A2 = A.reshape(P, M, K).copy()
    B2 = B.reshape(P, K, N).copy()
    for p in range(P):
        for rb in range(M // 128):
            for kb in range(K // 128):
                A2[p, rb * 128:(rb + 1) * 128, kb * 128:(kb + 1) * 128] *= np.float32(2.0 ** ((kb * (rb + 1) + p) % 4 - 2))
        for cb in range(N // 128):
            for kb in range(K // 128):
                if (kb + cb + p) % 3 == 0:
                    B2[p, kb * 128:(kb + 1) * 128, cb * 128:(cb + 1) * 128] *= np.float32(0.5)
    A2, B2 = A2.ravel(), B2.ravel()
    ws = _prepare(cuda, A2, B2, M, N, K, 0, 0, P)
    qa, qb, sa, sb = _ws_views(ws, M, N, K, P)
    C = torch.full((P * M * N,), float("nan"), device=cuda)
    g.matmul_tc_run(ws, M, N, K, C, engine="tc_fp8", batch=P)
    torch.cuda.synchronize()
    assert g.device_faults() == 0
    ref = oracle.matmul_fp8_dequant(qa, sa, qb, sb, M, N, K, batch=P)
    assert oracle.normwise_error(C.cpu().numpy(), ref) <= PIPE_TOL


def test_segment_plan_across_bit_words(cuda):
    # 40 blocks of K: the plan's segment-start bits span two 32-bit words, and
    # the scales change right at the word boundary and inside both words
    import torch
    M, N, K = 256, 512, 40 * 128
    A, B = _operands(M, N, K, 1, seed=51)
    A2 = A.reshape(M, K).copy()
    for kb in (3, 31, 32, 33, 39):
        A2[:, kb * 128:(kb + 1) * 128] *= np.float32(4.0)
    A2 = A2.ravel()
    ws = _prepare(cuda, A2, B, M, N, K, 0, 0, 1)
    qa, qb, sa, sb = _ws_views(ws, M, N, K, 1)
    C = torch.full((M * N,), float("nan"), device=cuda)
    g.matmul_tc_run(ws, M, N, K, C, engine="tc_fp8")
    torch.cuda.synchronize()
    assert g.device_faults() == 0
    ref = oracle.matmul_fp8_dequant(qa, sa, qb, sb, M, N, K)
    assert oracle.normwise_error(C.cpu().numpy(), ref) <= PIPE_TOL
