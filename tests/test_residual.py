"""The device FP64 residual (gatlas_matmul_residual_f32) is the checker of
every full-size accuracy figure: it recomputes op(A)·op(B) in double on the
GPU and reduces ||C - Cref||_F, ||Cref||_F, max |C - Cref| and
sum |C - Cref| (the reference's absdiff, OCLAppUtil.hpp:212-264).  Here it
is itself checked against the host FP64 oracle (oracle_matmul_f32_acc64,
the reference's check loop KernelMatmulBuffer.hpp:124-143 accumulated in
double) on every layout, with alpha, at ragged sizes up to 1024^3 and at
2048^3 for one layout."""
import numpy as np
import pytest

import gatlas_b200 as g
import oracle

pytestmark = pytest.mark.gpu


def _host_stats(C, ref):
    d = C.astype(np.float64) - ref
    return (np.sqrt(np.sum(d * d)), np.sqrt(np.sum(ref * ref)), np.max(np.abs(d)), np.sum(np.abs(d)))


def _check(cuda, M, N, K, ta, tb, alpha, seed, noise):
    import torch
    A = oracle.uniform(M * K, seed=seed)
    B = oracle.uniform(K * N, seed=seed + 1)
    ref = oracle.matmul(A, B, M, N, K, ta, tb, mode=oracle.F64, gemm=int(alpha != 1.0), alpha=alpha)
    # C: the float result of the fused chain, plus a seeded perturbation so
    # that the residual is far above the two FP64 products' own rounding
    C = oracle.matmul(A, B, M, N, K, ta, tb, mode=oracle.FMA, gemm=int(alpha != 1.0), alpha=alpha)
    if noise:
        C = (C + noise * oracle.uniform(M * N, seed=seed + 2)).astype(np.float32)
    t = lambda a: torch.from_numpy(a).to(cuda)
    got = g.residual(t(A), t(B), t(C), M, N, K, trans_a=ta, trans_b=tb, alpha=alpha)
    torch.cuda.synchronize()
    want = _host_stats(C, ref)
    # Cref differs between the two FP64 products by at most ~K*2^-53 relative;
    # with noise the differences dominate that by many orders of magnitude,
    # without it (C within ~1e-6 of Cref) the stats agree to ~1e-5 relative
    rtol = 1e-9 if noise else 1e-4
    assert got[1] == pytest.approx(want[1], rel=1e-12)
    for i in (0, 2, 3):
        assert got[i] == pytest.approx(want[i], rel=rtol), (i, got, want)
    return got, want


@pytest.mark.parametrize("ta,tb", [(0, 0), (1, 0), (0, 1), (1, 1)])
@pytest.mark.parametrize("M,N,K", [(1024, 1024, 1024), (1000, 777, 333), (33, 65, 1031)])
@pytest.mark.parametrize("alpha", [1.0, -0.75])
def test_residual_matches_host_fp64(cuda, ta, tb, M, N, K, alpha):
    _check(cuda, M, N, K, ta, tb, alpha, seed=M + N + K + 10 * ta + 20 * tb, noise=1e-3)


@pytest.mark.parametrize("ta,tb", [(0, 0), (1, 1)])
def test_residual_of_an_accurate_result(cuda, ta, tb):
    # C is the float FMA chain itself: errors near 1e-7 relative, the regime
    # of the accuracy figures the residual reports
    got, want = _check(cuda, 512, 640, 768, ta, tb, 1.0, seed=5, noise=0.0)
    assert got[0] / got[1] < 1e-5


def test_residual_2048_cubed(cuda):
    _check(cuda, 2048, 2048, 2048, 0, 0, 1.0, seed=77, noise=1e-4)


def test_residual_known_answer(cuda):
    # A = B = 1: Cref == K exactly, so a C equal to K gives a zero residual
    # and a C off by one in a single element gives exactly that
    import torch
    M, N, K = 300, 200, 100
    one = lambda n: torch.ones(n, device=cuda)
    C = torch.full((M * N,), float(K), device=cuda)
    assert g.residual(one(M * K), one(K * N), C, M, N, K) == (0.0, pytest.approx(K * np.sqrt(M * N)), 0.0, 0.0)
    C[1234] += 1.0
    r = g.residual(one(M * K), one(K * N), C, M, N, K)
    assert r[0] == 1.0 and r[2] == 1.0 and r[3] == 1.0
