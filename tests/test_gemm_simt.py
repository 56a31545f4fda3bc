"""SIMT SGEMM / DGEMM parity: bit-exact against the sequential fmaf chain
(oracle ORACLE_FMA) at every tuning point and layout; exact on the reference's
test pattern (C == K); FP64 residual at full size."""
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


def _mm(cuda, A, B, M, N, K, ta=0, tb=0, tile=None, gemm=False, Cin=None, alpha=1.0, beta=0.0,
        batch=1, engine="buffer"):
    import torch
    dt = torch.float32 if A.dtype == np.float32 else torch.float64
    C = _gpu(cuda, Cin) if Cin is not None else torch.full((batch * M * N,), float("nan"), dtype=dt, device=cuda)
    g.matmul(_gpu(cuda, A), _gpu(cuda, B), M, N, K, C=C, trans_a=ta, trans_b=tb, gemm=gemm,
             alpha=alpha, beta=beta, engine=engine, tile=tile, batch=batch)
    torch.cuda.synchronize()
    return C.cpu().numpy()


@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_golden_fixture(cuda, ta, tb):
    M, N, K = (int(v) for v in GOLDEN["mm_dims"])
    tag = f"mm_t{ta}{tb}"
    C = _mm(cuda, GOLDEN[f"{tag}_A"], GOLDEN[f"{tag}_B"], M, N, K, ta, tb)
    assert np.array_equal(C, GOLDEN[f"{tag}_fma"])
    C = _mm(cuda, GOLDEN[f"{tag}_A"], GOLDEN[f"{tag}_B"], M, N, K, ta, tb, gemm=True,
            Cin=GOLDEN[f"{tag}_Cin"], alpha=0.75, beta=-1.25)
    assert np.array_equal(C, GOLDEN[f"{tag}_gemm_fma"])


TUNING = [(gh, gw, bh, bw, vl) for gh in (8, 16) for gw in (8, 16) for bh in (4, 8)
          for bw in (4, 8) for vl in (1, 2, 4)]


@pytest.mark.parametrize("tile", TUNING, ids=lambda t: "x".join(map(str, t)))
def test_tuning_grid_bit_exact(cuda, tile):
    M, N, K = 128, 128, 96
    A = oracle.uniform(M * K, seed=1)
    B = oracle.uniform(K * N, seed=2)
    C = _mm(cuda, A, B, M, N, K, tile=tile)
    assert np.array_equal(C, oracle.matmul(A, B, M, N, K, mode=oracle.FMA))


@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("M,N,K", [(1, 1, 1), (7, 9, 11), (33, 65, 17), (129, 127, 64),
                                   (256, 200, 300), (64, 512, 1)])
def test_layouts_and_ragged_edges(cuda, ta, tb, M, N, K):
    A = oracle.uniform(M * K, seed=M + K)
    B = oracle.uniform(K * N, seed=N + K)
    C = _mm(cuda, A, B, M, N, K, ta, tb)
    assert np.array_equal(C, oracle.matmul(A, B, M, N, K, ta, tb, mode=oracle.FMA))


@pytest.mark.parametrize("ta,tb", [(0, 0), (1, 1)])
def test_known_answer_c_equals_k(cuda, ta, tb):
    M = N = K = 1024
    C = _mm(cuda, np.ones(M * K, np.float32), np.ones(K * N, np.float32), M, N, K, ta, tb)
    assert oracle.check_pattern(C, float(K))
    # GEMM test pattern: alpha = beta = 1 on a cleared C
    C = _mm(cuda, np.ones(M * K, np.float32), np.ones(K * N, np.float32), M, N, K, ta, tb,
            gemm=True, Cin=np.zeros(M * N, np.float32), alpha=1.0, beta=1.0)
    assert oracle.check_pattern(C, float(K))


def test_packed_batch_and_gemm(cuda):
    M, N, K, P = 64, 96, 80, 3
    A = oracle.uniform(P * M * K, seed=3)
    B = oracle.uniform(P * K * N, seed=4)
    Cin = oracle.uniform(P * M * N, seed=5)
    C = _mm(cuda, A, B, M, N, K, gemm=True, Cin=Cin, alpha=1.5, beta=-0.5, batch=P)
    ref = oracle.matmul(A, B, M, N, K, mode=oracle.FMA, gemm=1, Cin=Cin, alpha=1.5, beta=-0.5,
                        packed=P)
    assert np.array_equal(C, ref)


def test_beta_zero_does_not_read_c(cuda):
    M = N = K = 64
    A = oracle.uniform(M * K, seed=6)
    B = oracle.uniform(K * N, seed=7)
    Cin = np.full(M * N, np.nan, np.float32)
    C = _mm(cuda, A, B, M, N, K, gemm=True, Cin=Cin, alpha=2.0, beta=0.0)
    assert np.array_equal(C, oracle.matmul(A, B, M, N, K, mode=oracle.FMA, gemm=1,
                                           Cin=np.zeros_like(Cin), alpha=2.0, beta=0.0))


@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_dgemm_bit_exact(cuda, ta, tb):
    M, N, K = 96, 80, 72
    A = oracle.uniform(M * K, seed=8, dtype=np.float64)
    B = oracle.uniform(K * N, seed=9, dtype=np.float64)
    C = _mm(cuda, A, B, M, N, K, ta, tb)
    assert np.array_equal(C, oracle.matmul(A, B, M, N, K, ta, tb, mode=oracle.FMA, dtype=np.float64))


def test_unsupported_point_reports(cuda):
    # a vector width of 3 divides no K step: no kernel can be built for it
    with pytest.raises(g.GatlasError) as e:
        _mm(cuda, np.ones(36, np.float32), np.ones(36, np.float32), 6, 6, 6, tile=(8, 8, 4, 4, 3))
    assert e.value.status in (g.ERR_UNSUPPORTED, g.ERR_INVALID)


@pytest.mark.parametrize("ta,tb", [(0, 0), (1, 0), (0, 1), (1, 1)])
@pytest.mark.parametrize("tile", [(10, 10, 8, 4, 4), (9, 9, 4, 4, 4), (8, 8, 10, 1, 1), (10, 10, 12, 2, 2)])
def test_run_time_compiled_points_bit_exact(cuda, ta, tb, tile):
    # points of the reference's space outside the prebuilt grid (odd work
    # groups, blockings up to 12) are compiled with NVRTC on first use
    gh, gw, bh, bw, vl = tile
    if ta and (gh * bh) % vl:
        pytest.skip("not a valid point for transposed A")
    M, N, K = gh * bh * 2, gw * bw * 3, 72
    A = oracle.uniform(M * K, seed=gh + bh)
    B = oracle.uniform(K * N, seed=gw + bw)
    C = _mm(cuda, A, B, M, N, K, ta, tb, tile=tile)
    assert np.array_equal(C, oracle.matmul(A, B, M, N, K, ta, tb, mode=oracle.FMA))


def test_full_size_residual_4096(cuda):
    # FP64 residual on the device against the normwise tolerance 4*K*u
    import torch
    M = N = K = 4096
    A = torch.empty(M * K, dtype=torch.float32, device=cuda)
    B = torch.empty(K * N, dtype=torch.float32, device=cuda)
    g.fill(A, "uniform", seed=1)
    g.fill(B, "uniform", seed=2)
    C = g.matmul(A, B, M, N, K)
    fro, ref, mx, s1 = g.residual(A, B, C, M, N, K)
    assert fro / ref <= 4 * K * U32
    # and a sampled bit-exact check against the fmaf chain
    rows = [0, 1, 2047, 4095]
    Ah = A.view(M, K)[rows].cpu().numpy().ravel()
    ref_rows = oracle.matmul(Ah, B.cpu().numpy(), len(rows), N, K, mode=oracle.FMA)
    assert np.array_equal(C.view(M, N)[rows].cpu().numpy().ravel(), ref_rows)


# ---- image engine: SIMT math on TMA tensor-map tiles ------------------------------

IMAGE_TILES = [(16, 16, 8, 8), (16, 16, 8, 4), (8, 8, 8, 4), (16, 16, 4, 4), (8, 8, 4, 4)]


@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("tile", IMAGE_TILES, ids=lambda t: "x".join(map(str, t)))
def test_image_engine_bit_exact(cuda, ta, tb, tile):
    M, N, K = 256, 192, 100
    A = oracle.uniform(M * K, seed=sum(tile) + ta)
    B = oracle.uniform(K * N, seed=sum(tile) + 7 * tb)
    C = _mm(cuda, A, B, M, N, K, ta, tb, tile=tile + (0,), engine="image")
    assert np.array_equal(C, oracle.matmul(A, B, M, N, K, ta, tb, mode=oracle.FMA))
    assert g.device_faults() == 0


@pytest.mark.parametrize("ta,tb", [(0, 0), (1, 1)])
@pytest.mark.parametrize("M,N,K", [(4, 4, 4), (36, 68, 33), (130, 260, 64), (3520 // 10, 3520 // 10, 3520 // 10)])
def test_image_engine_ragged(cuda, ta, tb, M, N, K):
    # rows need 16-byte alignment for TMA: the stored inner dimensions are multiples of 4 here
    if (K if not ta else M) % 4 or (N if not tb else K) % 4:
        pytest.skip("TMA needs 16-byte aligned rows")
    A = oracle.uniform(M * K, seed=M)
    B = oracle.uniform(K * N, seed=N)
    C = _mm(cuda, A, B, M, N, K, ta, tb, engine="image")
    assert np.array_equal(C, oracle.matmul(A, B, M, N, K, ta, tb, mode=oracle.FMA))


def test_image_engine_gemm_batch_and_known_answer(cuda):
    M, N, K, P = 128, 128, 96, 2
    A = oracle.uniform(P * M * K, seed=3)
    B = oracle.uniform(P * K * N, seed=4)
    Cin = oracle.uniform(P * M * N, seed=5)
    C = _mm(cuda, A, B, M, N, K, gemm=True, Cin=Cin, alpha=0.5, beta=2.0, batch=P, engine="image")
    assert np.array_equal(C, oracle.matmul(A, B, M, N, K, mode=oracle.FMA, gemm=1, Cin=Cin, alpha=0.5, beta=2.0,
                                           packed=P))
    C = _mm(cuda, np.ones(512 * 512, np.float32), np.ones(512 * 512, np.float32), 512, 512, 512, engine="image")
    assert oracle.check_pattern(C, 512.0)


@pytest.mark.parametrize("tile", [(16, 16, 12, 4), (9, 9, 4, 4), (10, 10, 8, 4)])
def test_image_engine_run_time_compiled(cuda, tile):
    gh, gw, bh, bw = tile
    M, N, K = gh * bh * 2, gw * bw * 2, 64
    A = oracle.uniform(M * K, seed=11)
    B = oracle.uniform(K * N, seed=12)
    C = _mm(cuda, A, B, M, N, K, tile=tile + (0,), engine="image")
    assert np.array_equal(C, oracle.matmul(A, B, M, N, K, mode=oracle.FMA))


@pytest.mark.parametrize("ta,tb", [(0, 0), (1, 0)])
def test_image_engine_double(cuda, ta, tb):
    M, N, K = 128, 96, 80
    A = oracle.uniform(M * K, seed=8, dtype=np.float64)
    B = oracle.uniform(K * N, seed=9, dtype=np.float64)
    C = _mm(cuda, A, B, M, N, K, ta, tb, engine="image")
    assert np.array_equal(C, oracle.matmul(A, B, M, N, K, ta, tb, mode=oracle.FMA, dtype=np.float64))


def test_image_engine_empty_contraction_and_unaligned_rows(cuda):
    M, N = 64, 64
    Cin = oracle.uniform(M * N, seed=21)
    C = _mm(cuda, np.zeros(0, np.float32), np.zeros(0, np.float32), M, N, 0, gemm=True, Cin=Cin, alpha=1.0,
            beta=0.5, engine="image")
    assert np.array_equal(C, oracle.matmul(np.zeros(0, np.float32), np.zeros(0, np.float32), M, N, 0, mode=oracle.FMA,
                                           gemm=1, Cin=Cin, alpha=1.0, beta=0.5))
    # K = 30 gives A rows of 120 bytes: TMA needs 16-byte aligned rows, the engine refuses
    A = oracle.uniform(M * 30, seed=1)
    B = oracle.uniform(30 * N, seed=2)
    with pytest.raises(RuntimeError, match="16-byte"):
        _mm(cuda, A, B, M, N, 30, engine="image")


@pytest.mark.parametrize("tile", [(8, 16, 8, 8, 2), (16, 8, 8, 8, 2), (8, 8, 8, 8, 2), (16, 16, 8, 8, 2), (0, 0, 0, 0, 0)],
                         ids=lambda t: "x".join(map(str, t)))
@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_dgemm_points_bit_exact(cuda, tile, ta, tb):
    M, N, K = 200, 136, 72
    A = oracle.uniform(M * K, seed=18, dtype=np.float64)
    B = oracle.uniform(K * N, seed=19, dtype=np.float64)
    C = _mm(cuda, A, B, M, N, K, ta, tb, tile=tile + (0,) if any(tile) else None)
    assert np.array_equal(C, oracle.matmul(A, B, M, N, K, ta, tb, mode=oracle.FMA, dtype=np.float64))
