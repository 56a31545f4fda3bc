"""The oracle pinned against the reference itself.

oracle/_ref holds the reference's own generated kernels -- emitted by the
reference's generators from its sources (KernelMatmulBuffer.hpp:174-342,
KernelMatmulImage.hpp:190-314, KernelMatvecBuffer.hpp:180-325,
KernelMatvecImage.hpp:185-297, KernelSaxpyBuffer.hpp:143-225) and compiled
for the host CPU by oracle/ref (see gen_kernels.py).  OpenCL leaves the
rounding of mad() to the implementation, so each kernel is built twice:

- mad fused: bit-exact against the oracle's ORACLE_FMA restatement, the
  contract the GPU engines are held to;
- mad rounded as a product and a sum: bit-exact against ORACLE_REFHOST, the
  reference's host check loops (KernelMatmulBuffer.hpp:124-143,
  KernelMatvecBuffer.hpp:122-138, KernelSaxpyBuffer.hpp:118-120).

So on these inputs the oracle computes exactly what the reference's kernels
compute.  The image SAXPY kernel is not built: its 2-D form indexes texels by
scalar counts and reads past the image (KernelSaxpyImage.hpp:210-227), and
its 1-D form needs an image n/4 texels high.
"""
import numpy as np
import pytest

import oracle

R = pytest.importorskip("oracle.ref")

if not R.available() and not R.sources_present():
    pytest.skip("oracle/_ref is not built and the reference's sources are absent", allow_module_level=True)

PARITY = [k for k in R.kernels() if not k.startswith("bench_")]


def _dtype(k):
    return np.float64 if k["scalar"] == "double" else np.float32


def _case(kid, fused, alpha=0.75, beta=-1.25, dist="uniform"):
    k = R.kernel(kid)
    op, p, dt = k["op"], k["params"], _dtype(k)
    mode = oracle.FMA if fused else oracle.REFHOST
    gen = (lambda n, s: oracle.uniform(n, seed=s, dtype=dt)) if dist == "uniform" else \
        (lambda n, s: oracle.pow2(n, seed=s).astype(dt))
    if op == "matmul":
        P, gemm, M, N, K, ta, tb = p[:7]
        A, B, C0 = gen(P * M * K, 11), gen(P * K * N, 12), gen(P * M * N, 13)
        C = C0.copy()
        R.run(kid, A, B, C, alpha, beta, fused=fused)
        want = oracle.matmul(A, B, M, N, K, ta, tb, mode=mode, gemm=gemm, Cin=C0, alpha=alpha, beta=beta,
                             packed=P, dtype=dt)
    elif op == "matvec":
        P, gemv, M, N, ta = p[:5]
        A, x, y0 = gen(P * M * N, 21), gen(P * N, 22), gen(P * M, 23)
        C = y0.copy()
        R.run(kid, A, x, C, alpha, beta, fused=fused)
        want = oracle.matvec(A, x, M, N, ta, mode=mode, gemv=gemv, cin=y0, alpha=alpha, beta=beta, packed=P,
                             dtype=dt)
    else:
        P, M, N = p[:3]
        X, Y = gen(P * M * N, 31), gen(P * M * N, 32)
        C = np.empty_like(X)
        R.run(kid, X, Y, C, alpha, fused=fused)
        want = oracle.saxpy(alpha, X, Y, mode=mode, dtype=dt)
    return C, want


@pytest.mark.parametrize("fused", [True, False], ids=["mad_fused", "mad_separate"])
@pytest.mark.parametrize("kid", PARITY)
def test_oracle_equals_reference_kernel(kid, fused):
    got, want = _case(kid, fused)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("kid", ["mm_f4_nn", "mm_img_f_tn_gemm", "mv_f4_t_gemv", "sx_f4_2d"])
def test_oracle_equals_reference_kernel_on_powers_of_two(kid):
    # sign * 2^e operands (the precision workload's second distribution)
    got, want = _case(kid, True, alpha=1.0, beta=0.5, dist="pow2")
    assert np.array_equal(got, want)


def test_the_two_roundings_of_mad_differ():
    # the builds really differ: uniform operands part in the last bits
    f, _ = _case("mm_f4_nn", True)
    s, _ = _case("mm_f4_nn", False)
    assert not np.array_equal(f, s)


@pytest.mark.parametrize("kid", ["mm_f4_nn", "mm_f1", "mm_img_f_nn", "mv_f4_n", "sx_f4_1d"])
def test_reference_known_answers(kid):
    # the reference's test pattern: A = B = 1 gives C == K (matmul), c == N
    # (matvec); x = y = 1, alpha = 1 gives z == 2 (KernelMatmulBuffer.hpp:77-79,
    # KernelMatvecBuffer.hpp:76-77, KernelSaxpyBuffer.hpp:80)
    k = R.kernel(kid)
    op, p = k["op"], k["params"]
    if op == "matmul":
        P, _, M, N, K = p[:5]
        C = np.zeros(P * M * N, np.float32)
        R.run(kid, np.ones(P * M * K, np.float32), np.ones(P * K * N, np.float32), C)
        assert oracle.check_pattern(C, float(K))
    elif op == "matvec":
        P, _, M, N = p[:4]
        C = np.zeros(P * M, np.float32)
        R.run(kid, np.ones(P * M * N, np.float32), np.ones(P * N, np.float32), C)
        assert oracle.check_pattern(C, float(N))
    else:
        n = p[0] * p[1] * p[2]
        C = np.zeros(n, np.float32)
        R.run(kid, np.ones(n, np.float32), np.ones(n, np.float32), C, 1.0)
        assert oracle.check_pattern(C, 2.0)


def test_workload_kernel_on_a_band_of_work_groups():
    # the 8192^3 buffer kernel that the CPU baseline samples: one band of work
    # groups (128 rows of C) equals the oracle's fused chain on those rows
    kid = "bench_sgemm_8192"
    M = N = K = 8192
    k = R.kernel(kid)
    rows = k["local"][1] * (k["params"][9])  # work-group height x inner blocking height
    A = oracle.uniform(M * K, seed=41)
    B = oracle.uniform(K * N, seed=42)
    C = np.zeros(M * N, np.float32)
    R.run(kid, A, B, C, group_begin=(0, 3), group_end=(0, 4))
    band = slice(3 * rows * N, 4 * rows * N)
    want = oracle.matmul(A[3 * rows * K: 4 * rows * K], B, rows, N, K, mode=oracle.FMA)
    assert np.array_equal(C[band], want)
    assert not C[: 3 * rows * N].any() and not C[4 * rows * N:].any()
