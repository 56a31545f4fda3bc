"""The GPU engines against the reference's own generated kernels.

Each case runs the reference's kernel for one parameter point on the host
CPU (oracle/_ref, built from the reference's sources; its mad fused, the
rounding the engines are held to) and the library's engine for the same
point on the GPU, on the same seeded inputs: SGEMM/DGEMM and SAXPY are
bit-exact, GEMV (whose GPU reduction order differs from the reference's
sequential loop) within the normwise 4*N*u of the other GEMV tests.
"""
import numpy as np
import pytest

import gatlas_b200 as g
import oracle

R = pytest.importorskip("oracle.ref")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not R.available(), reason="oracle/_ref (the reference's kernels) is not built")]


def _t(cuda, a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


def _matmul_case(cuda, kid, engine):
    import torch
    k = R.kernel(kid)
    P, gemm, M, N, K, ta, tb, gh, gw, bh, bw, x = k["params"]
    dt = np.float64 if k["scalar"] == "double" else np.float32
    A = oracle.uniform(P * M * K, seed=51, dtype=dt)
    B = oracle.uniform(P * K * N, seed=52, dtype=dt)
    C0 = oracle.uniform(P * M * N, seed=53, dtype=dt)
    want = R.run(kid, A, B, C0.copy(), 0.75, -1.25, fused=True)
    vl = bw
    Cd = _t(cuda, C0)
    g.matmul(_t(cuda, A), _t(cuda, B), M, N, K, C=Cd, trans_a=ta, trans_b=tb, gemm=gemm, alpha=0.75, beta=-1.25,
             engine=engine, tile=(gh, gw, bh, bw, vl, x), batch=P)
    torch.cuda.synchronize()
    assert g.device_faults() == 0
    return Cd.cpu().numpy(), want


@pytest.mark.parametrize("kid", ["mm_f4_nn", "mm_f4_tn", "mm_f4_nt", "mm_f4_tt_gemm_p2", "mm_f2_gemm", "mm_f1",
                                 "mm_d2_gemm", "bench_sgemm_1024"])
def test_buffer_engine_equals_reference_kernel(cuda, kid):
    got, want = _matmul_case(cuda, kid, "buffer")
    assert np.array_equal(got, want)


@pytest.mark.parametrize("kid", ["mm_img_f_nn", "mm_img_f_tn_gemm", "mm_img_d"])
def test_image_engine_equals_reference_kernel(cuda, kid):
    got, want = _matmul_case(cuda, kid, "image")
    assert np.array_equal(got, want)


@pytest.mark.parametrize("engine", ["buffer", "image"])
def test_saxpy_full_size_equals_reference_kernel(cuda, engine):
    # n = 2^28, the memory-bound workload's size
    import torch
    n = 1 << 28
    X = oracle.uniform(n, seed=61)
    Y = oracle.uniform(n, seed=62)
    want = R.run("bench_saxpy_2p28", X, Y, np.empty_like(X), 0.5, fused=True)
    z = g.saxpy(0.5, _t(cuda, X), _t(cuda, Y), engine=engine)
    torch.cuda.synchronize()
    assert np.array_equal(z.cpu().numpy(), want)


@pytest.mark.parametrize("kid,engine", [("bench_sgemv_n_16384", "buffer"), ("bench_sgemv_t_16384", "buffer"),
                                        ("bench_sgemv_img_n_16384", "image"), ("bench_sgemv_img_t_16384", "image")])
def test_gemv_full_size_against_reference_kernel(cuda, kid, engine):
    import torch
    k = R.kernel(kid)
    _, _, M, N, ta = k["params"][:5]
    A = oracle.uniform(M * N, seed=71)
    x = oracle.uniform(N, seed=72)
    want = R.run(kid, A, x, np.zeros(M, np.float32), fused=True)
    y = g.matvec(_t(cuda, A), _t(cuda, x), M, N, trans_a=ta, engine=engine)
    torch.cuda.synchronize()
    exact = oracle.matvec(A, x, M, N, ta, mode=oracle.F64)
    assert oracle.normwise_error(y.cpu().numpy(), want) <= 4 * N * 2.0 ** -24
    assert oracle.normwise_error(want, exact) <= 4 * N * 2.0 ** -24
