"""GEMV parity: within the normwise tolerance 4*N*u of the FP64 oracle, exact
on the reference's test pattern (c == N)."""
import os

import numpy as np
import pytest

import gatlas_b200 as g
import oracle

pytestmark = pytest.mark.gpu
GOLDEN = np.load(os.path.join(os.path.dirname(__file__), "golden", "oracle_small.npz"))
U32 = 2.0 ** -24


def _gpu(cuda, a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


def _matvec(cuda, A, x, M, N, ta, engine="buffer", gemv=False, yin=None, alpha=1.0, beta=0.0,
            batch=1):
    import torch
    y = _gpu(cuda, yin) if yin is not None else torch.zeros(batch * M, dtype=torch.float32, device=cuda)
    g.matvec(_gpu(cuda, A), _gpu(cuda, x), M, N, y=y, trans_a=ta, gemv=gemv, alpha=alpha,
             beta=beta, engine=engine, batch=batch)
    torch.cuda.synchronize()
    return y.cpu().numpy()


@pytest.mark.parametrize("ta", [0, 1])
def test_golden_fixture(cuda, ta):
    M, N = (int(v) for v in GOLDEN["mv_dims"])
    y = _matvec(cuda, GOLDEN[f"mv_t{ta}_A"], GOLDEN[f"mv_t{ta}_x"], M, N, ta)
    assert oracle.normwise_error(y, GOLDEN[f"mv_t{ta}_f64"]) <= 4 * N * U32
    y = _matvec(cuda, GOLDEN[f"mv_t{ta}_A"], GOLDEN[f"mv_t{ta}_x"], M, N, ta, gemv=True,
                yin=GOLDEN[f"mv_t{ta}_yin"], alpha=0.5, beta=2.0)
    assert oracle.normwise_error(y, GOLDEN[f"mv_t{ta}_gemv_f64"]) <= 4 * N * U32


@pytest.mark.parametrize("ta", [0, 1])
@pytest.mark.parametrize("M,N", [(64, 64), (1024, 4096), (4096, 1024), (16384, 512)])
def test_known_answer_c_equals_n(cuda, ta, M, N):
    y = _matvec(cuda, np.ones(M * N, np.float32), np.ones(N, np.float32), M, N, ta)
    assert oracle.check_pattern(y, float(N))


@pytest.mark.parametrize("ta", [0, 1])
@pytest.mark.parametrize("M,N", [(1, 1), (1, 37), (37, 1), (33, 65), (127, 129), (1000, 1001),
                                 (2048, 3072), (4099, 257), (301, 4096), (1001, 6000), (7, 10003), (3, 65536)])
def test_tolerance_vs_f64(cuda, ta, M, N):
    A = oracle.uniform(M * N, seed=M * 7 + N)
    x = oracle.uniform(N, seed=N * 3 + 1)
    y = _matvec(cuda, A, x, M, N, ta)
    ref = oracle.matvec(A, x, M, N, ta, mode=oracle.F64)
    assert oracle.normwise_error(y, ref) <= 4 * N * U32


@pytest.mark.parametrize("ta", [0, 1])
def test_gemv_alpha_beta_and_batch(cuda, ta):
    M, N, P = 300, 500, 3
    A = oracle.uniform(P * M * N, seed=1)
    x = oracle.uniform(P * N, seed=2)
    yin = oracle.uniform(P * M, seed=3)
    y = _matvec(cuda, A, x, M, N, ta, gemv=True, yin=yin, alpha=-0.5, beta=1.5, batch=P)
    ref = oracle.matvec(A, x, M, N, ta, mode=oracle.F64, gemv=1, cin=yin, alpha=-0.5, beta=1.5,
                        packed=P)
    assert oracle.normwise_error(y, ref) <= 4 * N * U32


@pytest.mark.parametrize("ta", [0, 1])
def test_deterministic(cuda, ta):
    M, N = 2048, 2048
    A = oracle.uniform(M * N, seed=5)
    x = oracle.uniform(N, seed=6)
    y1 = _matvec(cuda, A, x, M, N, ta)
    y2 = _matvec(cuda, A, x, M, N, ta)
    assert np.array_equal(y1, y2)


def test_empty_inner_dimension(cuda):
    # N == 0: y = alpha*0 + beta*y
    yin = oracle.uniform(64, seed=9)
    for ta in (0, 1):
        y = _matvec(cuda, np.zeros(1, np.float32), np.zeros(1, np.float32), 64, 0, ta, gemv=True,
                    yin=yin, alpha=2.0, beta=0.5)
        assert np.array_equal(y, (yin * np.float32(0.5)).astype(np.float32))


@pytest.mark.parametrize("ta", [0, 1])
def test_full_size_16384(cuda, ta):
    # full GEMV workload: A 16384^2 (1 GiB); checked against FP64 on 256 sampled rows
    import torch
    M = N = 16384
    A = torch.empty(M * N, dtype=torch.float32, device=cuda)
    x = torch.empty(N, dtype=torch.float32, device=cuda)
    g.fill(A, "uniform", seed=11)
    g.fill(x, "uniform", seed=12)
    y = g.matvec(A, x, M, N, trans_a=ta)
    torch.cuda.synchronize()
    rows = np.random.default_rng(0).choice(M, 256, replace=False)
    A64 = A.view(N, M).double() if ta else A.view(M, N).double()
    ref = (A64[:, rows].T if ta else A64[rows]) @ x.double()
    err = torch.linalg.norm(y[rows].double() - ref) / torch.linalg.norm(ref)
    assert float(err) <= 4 * N * U32


# ---- image engine (TMA tensor-map tiles) ----------------------------------------

@pytest.mark.parametrize("ta", [0, 1])
@pytest.mark.parametrize("M,N", [(4, 4), (16, 256), (100, 260), (1024, 4096), (4096, 1000), (333 * 4, 777 * 4),
                                 (16384, 512)])
def test_image_engine_tolerance(cuda, ta, M, N):
    A = oracle.uniform(M * N, seed=M + 13 * N)
    x = oracle.uniform(N, seed=N + 5)
    y = _matvec(cuda, A, x, M, N, ta, engine="image")
    ref = oracle.matvec(A, x, M, N, ta, mode=oracle.F64)
    assert oracle.normwise_error(y, ref) <= 4 * N * U32


@pytest.mark.parametrize("ta", [0, 1])
def test_image_engine_known_answer_and_gemv(cuda, ta):
    M, N = 2048, 4096
    y = _matvec(cuda, np.ones(M * N, np.float32), np.ones(N, np.float32), M, N, ta, engine="image")
    assert oracle.check_pattern(y, float(N))
    A = oracle.uniform(M * N, seed=21)
    x = oracle.uniform(N, seed=22)
    yin = oracle.uniform(M, seed=23)
    y = _matvec(cuda, A, x, M, N, ta, engine="image", gemv=True, yin=yin, alpha=1.5, beta=-0.25)
    ref = oracle.matvec(A, x, M, N, ta, mode=oracle.F64, gemv=1, cin=yin, alpha=1.5, beta=-0.25)
    assert oracle.normwise_error(y, ref) <= 4 * N * U32


def test_image_engine_rejects_unaligned_rows(cuda):
    with pytest.raises(g.GatlasError) as e:
        _matvec(cuda, np.ones(33 * 65, np.float32), np.ones(65, np.float32), 33, 65, 0, engine="image")
    assert e.value.status == g.ERR_UNSUPPORTED
    assert g.device_faults() == 0


@pytest.mark.parametrize("ta", [0, 1])
def test_image_engine_full_size_matches_buffer(cuda, ta):
    import torch
    M = N = 16384
    A = torch.empty(M * N, dtype=torch.float32, device=cuda)
    x = torch.empty(N, dtype=torch.float32, device=cuda)
    g.fill(A, "uniform", seed=31)
    g.fill(x, "uniform", seed=32)
    yb = g.matvec(A, x, M, N, trans_a=ta, engine="buffer")
    yi = g.matvec(A, x, M, N, trans_a=ta, engine="image")
    torch.cuda.synchronize()
    err = torch.linalg.norm((yi - yb).double()) / torch.linalg.norm(yb.double())
    assert float(err) <= 4 * N * U32
    assert g.device_faults() == 0


@pytest.mark.parametrize("engine", ["buffer", "image"])
@pytest.mark.parametrize("M,N", [(16384, 16384), (4096, 50000), (300, 7000), (1024, 96)])
def test_workspace_of_the_queried_size_fits(cuda, engine, M, N):
    """A workspace of exactly gatlas_matvec_workspace_size bytes is accepted by
    both engines' column-major paths, and gives the same y as library scratch."""
    import torch
    A = torch.empty(M * N, dtype=torch.float32, device=cuda)
    x = torch.empty(N, dtype=torch.float32, device=cuda)
    g.fill(A, "uniform", seed=M + N)
    g.fill(x, "uniform", seed=N + 3)
    need = g.matvec_workspace_size(M, N, trans_a=True)
    ws = torch.empty(max(need, 1), dtype=torch.uint8, device=cuda)[:need]
    y_ws = g.matvec(A, x, M, N, trans_a=True, engine=engine, workspace=ws if need else None)
    y_lib = g.matvec(A, x, M, N, trans_a=True, engine=engine)
    torch.cuda.synchronize()
    assert torch.equal(y_ws, y_lib)
    lo = max(0, M - 48)
    Aw = A.view(N, M)[:, lo:].contiguous().cpu().numpy().ravel()
    ref = oracle.matvec(Aw, x.cpu().numpy(), M - lo, N, 1, mode=oracle.F64)
    assert oracle.normwise_error(y_ws[lo:].cpu().numpy(), ref) <= 4 * N * U32
    assert g.device_faults() == 0


def _exact_matvec(A, x, M, N, ta, gemv=False, yin=None, alpha=1.0, beta=0.0):
    """y in extended precision (numpy longdouble) from the float64 operands:
    the reference's host loop (KernelMatvecBuffer.hpp:122-138) evaluated
    without its own rounding, as the yardstick for both float64 results."""
    Al = np.asarray(A, dtype=np.longdouble).reshape((N, M) if ta else (M, N))
    Al = Al.T if ta else Al
    y = Al @ np.asarray(x, dtype=np.longdouble)
    if gemv:
        y = alpha * y + beta * np.asarray(yin, dtype=np.longdouble)
    return y


DGEMV_CASES = [("buffer", 999, 777), ("buffer", 1000, 778), ("image", 1000, 778), ("buffer", 4096, 4096),
               ("image", 4096, 4096), ("buffer", 334, 20000), ("image", 334, 20000), ("buffer", 20000, 64),
               ("image", 20000, 64)]


@pytest.mark.parametrize("ta", [0, 1])
@pytest.mark.parametrize("engine,M,N", DGEMV_CASES)
def test_dgemv_vs_oracle(cuda, ta, engine, M, N):
    """gatlas_matvec_f64 on both layouts and both engines (the image engine
    is the reference's doubleimg matvec, KernelMatvecImage.hpp:61-65) against
    the oracle's float64 host loop (mode FMA, sequential k) and an
    extended-precision product: both within 4*N*u of the exact value,
    normwise, with u = 2^-53."""
    U64 = 2.0 ** -53
    A = oracle.uniform(M * N, seed=M + 3 * N + ta, dtype=np.float64)
    x = oracle.uniform(N, seed=N + 5, dtype=np.float64)
    y = _matvec_f64(cuda, A, x, M, N, ta, engine=engine)
    exact = _exact_matvec(A, x, M, N, ta)
    host = oracle.matvec(A, x, M, N, ta, mode=oracle.FMA, dtype=np.float64)
    assert _normwise(y, exact) <= 4 * N * U64
    assert _normwise(host, exact) <= 4 * N * U64
    assert _normwise(y, host) <= 8 * N * U64
    # the general form with alpha and beta
    yin = oracle.uniform(M, seed=M + 9, dtype=np.float64)
    y = _matvec_f64(cuda, A, x, M, N, ta, gemv=True, yin=yin, alpha=0.75, beta=-2.0, engine=engine)
    assert _normwise(y, _exact_matvec(A, x, M, N, ta, True, yin, 0.75, -2.0)) <= 4 * N * U64


@pytest.mark.parametrize("engine", ["buffer", "image"])
@pytest.mark.parametrize("ta", [0, 1])
def test_dgemv_known_answer(cuda, ta, engine):
    M, N = 778, 1032
    y = _matvec_f64(cuda, np.ones(M * N), np.ones(N), M, N, ta, engine=engine)
    assert np.all(y == N)


@pytest.mark.parametrize("ta", [0, 1])
def test_double_image_engine_full_size_matches_buffer(cuda, ta):
    # 16384^2 doubles (2 GiB): the image engine against the buffer engine
    import torch
    M = N = 16384
    A = torch.empty(M * N, dtype=torch.float64, device=cuda)
    x = torch.empty(N, dtype=torch.float64, device=cuda)
    g.fill(A, "uniform", seed=33)
    g.fill(x, "uniform", seed=34)
    yb = g.matvec(A, x, M, N, trans_a=ta, engine="buffer")
    yi = g.matvec(A, x, M, N, trans_a=ta, engine="image")
    torch.cuda.synchronize()
    err = torch.linalg.norm(yi - yb) / torch.linalg.norm(yb)
    assert float(err) <= 4 * N * 2.0 ** -53
    assert g.device_faults() == 0


def test_double_image_engine_rejects_odd_rows(cuda):
    with pytest.raises(g.GatlasError) as e:
        _matvec_f64(cuda, np.ones(33 * 65), np.ones(65), 33, 65, 0, engine="image")
    assert e.value.status == g.ERR_UNSUPPORTED


def _normwise(y, ref):
    ref = np.asarray(ref, dtype=np.longdouble)
    d = np.asarray(y, dtype=np.longdouble) - ref
    return float(np.sqrt(np.sum(d * d)) / np.sqrt(np.sum(ref * ref)))


def _matvec_f64(cuda, A, x, M, N, ta, gemv=False, yin=None, alpha=1.0, beta=0.0, engine="buffer"):
    import torch
    y = _gpu(cuda, yin) if yin is not None else torch.zeros(M, dtype=torch.float64, device=cuda)
    g.matvec(_gpu(cuda, np.asarray(A, np.float64)), _gpu(cuda, np.asarray(x, np.float64)), M, N, y=y,
             trans_a=ta, gemv=gemv, alpha=alpha, beta=beta, engine=engine)
    torch.cuda.synchronize()
    assert g.device_faults() == 0
    return y.cpu().numpy()
