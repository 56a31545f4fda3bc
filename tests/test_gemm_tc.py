"""Tensor-core engines (tcgen05): BF16 in / FP32 out, and FP32 operands split
into BF16 pieces (3 or 6 products).  Checked against the FP64 oracle: exact on
the reference's test pattern (C == K), within each engine's error budget on
uniform[-1,1) inputs, and within 4*K*u when every product is exact (sign*2^e
inputs, where the BF16 pieces represent the operands exactly)."""
import ctypes

import numpy as np
import pytest

import gatlas_b200 as g
import oracle

pytestmark = pytest.mark.gpu
U32 = 2.0 ** -24
ENGINES = ["tc_bf16", "tc_split3", "tc_split6"]
# normwise error budgets vs FP64 on uniform[-1,1) operands, K <= 1024
# BF16 rounds each operand with unit roundoff 2^-8, so one product can be off by 2^-7
BUDGET = {"tc_bf16": 2.0 ** -7, "tc_split3": 8e-6, "tc_split6": 2.5e-6}


def _gpu(cuda, a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


def _mm(cuda, A, B, M, N, K, engine, ta=0, tb=0, gemm=False, Cin=None, alpha=1.0, beta=0.0, batch=1):
    import torch
    C = _gpu(cuda, Cin) if Cin is not None else torch.full((batch * M * N,), float("nan"), device=cuda)
    g.matmul(_gpu(cuda, A), _gpu(cuda, B), M, N, K, C=C, trans_a=ta, trans_b=tb, gemm=gemm,
             alpha=alpha, beta=beta, engine=engine, batch=batch)
    torch.cuda.synchronize()
    assert g.device_faults() == 0
    return C.cpu().numpy()


@pytest.mark.parametrize("engine", ENGINES)
def test_known_answer_c_equals_k(cuda, engine):
    M = N = K = 1024
    C = _mm(cuda, np.ones(M * K, np.float32), np.ones(K * N, np.float32), M, N, K, engine)
    assert oracle.check_pattern(C, float(K))


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("M,N,K", [(128, 256, 32), (200, 300, 100), (257, 129, 520), (64, 1000, 8),
                                   (1, 1, 1), (512, 512, 1024)])
def test_uniform_within_budget(cuda, engine, ta, tb, M, N, K):
    A = oracle.uniform(M * K, seed=M + 3 * K)
    B = oracle.uniform(K * N, seed=N + 5 * K)
    C = _mm(cuda, A, B, M, N, K, engine, ta, tb)
    ref = oracle.matmul(A, B, M, N, K, ta, tb, mode=oracle.F64)
    assert oracle.normwise_error(C, ref) <= BUDGET[engine]


@pytest.mark.parametrize("engine", ENGINES)
def test_exact_products_meet_fp32_tolerance(cuda, engine):
    M, N, K = 256, 512, 512
    A = oracle.pow2(M * K, seed=1)
    B = oracle.pow2(K * N, seed=2)
    C = _mm(cuda, A, B, M, N, K, engine)
    ref = oracle.matmul(A, B, M, N, K, mode=oracle.F64)
    assert oracle.normwise_error(C, ref) <= 4 * K * U32


@pytest.mark.parametrize("engine", ENGINES)
def test_gemm_alpha_beta_batch(cuda, engine):
    M, N, K, P = 160, 272, 96, 3
    A = oracle.uniform(P * M * K, seed=7)
    B = oracle.uniform(P * K * N, seed=8)
    Cin = oracle.uniform(P * M * N, seed=9)
    C = _mm(cuda, A, B, M, N, K, engine, gemm=True, Cin=Cin, alpha=0.5, beta=-2.0, batch=P)
    ref = oracle.matmul(A, B, M, N, K, mode=oracle.F64, gemm=1, Cin=Cin, alpha=0.5, beta=-2.0,
                        packed=P)
    assert oracle.normwise_error(C, ref) <= BUDGET[engine]


@pytest.mark.parametrize("engine", ENGINES)
def test_caller_workspace(cuda, engine):
    import torch
    M, N, K = 256, 256, 256
    ws = torch.empty(g.matmul_workspace_size(M, N, K, engine) + 1024, dtype=torch.uint8, device=cuda)
    A = oracle.uniform(M * K, seed=1)
    B = oracle.uniform(K * N, seed=2)
    C = g.matmul(_gpu(cuda, A), _gpu(cuda, B), M, N, K, engine=engine, workspace=ws)
    torch.cuda.synchronize()
    ref = oracle.matmul(A, B, M, N, K, mode=oracle.F64)
    assert oracle.normwise_error(C.cpu().numpy(), ref) <= BUDGET[engine]
    with pytest.raises(g.GatlasError):
        g.matmul(_gpu(cuda, A), _gpu(cuda, B), M, N, K, engine=engine, workspace=ws[:1024])


def test_empty_k(cuda):
    Cin = oracle.uniform(64 * 64, seed=3)
    C = _mm(cuda, np.zeros(1, np.float32), np.zeros(1, np.float32), 64, 64, 0, "tc_split3",
            gemm=True, Cin=Cin, alpha=1.0, beta=0.5)
    assert np.array_equal(C, (Cin * np.float32(0.5)).astype(np.float32))


@pytest.mark.parametrize("dist", ["uniform", "pow2"])
def test_full_size_split6_matches_simt_error(cuda, dist):
    # 4096^3 on the device: split-BF16 with six products and promoted
    # accumulation is at least as accurate as the SIMT FP32 fmaf chain, and
    # three products stay within twice the two-piece representation limit
    import torch
    M = N = K = 4096
    A = torch.empty(M * K, device=cuda)
    B = torch.empty(K * N, device=cuda)
    g.fill(A, dist, seed=1)
    g.fill(B, dist, seed=2)
    errs = {}
    for eng in ("buffer", "tc_split3", "tc_split6"):
        C = g.matmul(A, B, M, N, K, engine=eng)
        fro, ref, _, _ = g.residual(A, B, C, M, N, K)
        errs[eng] = fro / ref
    assert errs["tc_split6"] <= errs["buffer"] * 1.05
    assert errs["tc_split3"] <= (8e-6 if dist == "uniform" else errs["buffer"] * 1.05)


def test_promotion_interval_is_selectable(cuda):
    import ctypes
    M, N, K = 256, 256, 2048
    A = oracle.uniform(M * K, seed=4)
    B = oracle.uniform(K * N, seed=5)
    ref = oracle.matmul(A, B, M, N, K, mode=oracle.F64)
    At, Bt = _gpu(cuda, A), _gpu(cuda, B)
    errs = []
    for extra in (1, 4, 64):
        import torch
        C = torch.empty(M * N, device=cuda)
        d = g.matmul_desc(M, N, K, engine="tc_split6", tile=(0, 0, 0, 0, 0, extra))
        g.check(g.lib().gatlas_matmul_f32(ctypes.byref(d), g._ptr(At), g._ptr(Bt), g._ptr(C), None, 0,
                                          g._stream()))
        torch.cuda.synchronize()
        errs.append(oracle.normwise_error(C.cpu().numpy(), ref))
    assert errs[0] <= errs[2] and errs[1] <= errs[2]


@pytest.mark.parametrize("engine", ENGINES + ["tc_fp8"])
@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("M,N,K", [(520, 300, 384), (256, 256, 4096), (129, 1000, 40)])
@pytest.mark.parametrize("beta", [0.5, 0.0])
def test_cta_pairs_match_single_ctas(cuda, engine, ta, tb, M, N, K, beta):
    # 256 x 256 tiles on CTA pairs (cta_group::2) and 128 x 256 tiles on single
    # CTAs run the same pieces through the same MMA order and promotion; beta = 0
    # stores C through TMA where C's rows are 16-byte aligned, beta != 0 reads it
    A = oracle.uniform(M * K, seed=M + K + ta)
    B = oracle.uniform(K * N, seed=N + K + tb)
    assert g.get_option("tc_pair") == 1
    try:
        g.set_option("tc_pair", 0)
        single = _mm(cuda, A, B, M, N, K, engine, ta, tb, gemm=True, Cin=oracle.uniform(M * N, seed=3),
                     alpha=1.5, beta=beta)
        g.set_option("tc_pair", 2)
        pair = _mm(cuda, A, B, M, N, K, engine, ta, tb, gemm=True, Cin=oracle.uniform(M * N, seed=3),
                   alpha=1.5, beta=beta)
    finally:
        g.set_option("tc_pair", 1)
    assert np.array_equal(single, pair)


@pytest.mark.parametrize("ta,tb", [(0, 0), (1, 1)])
@pytest.mark.parametrize("M,N,K,beta,batch", [(4000, 2500, 300, 0.0, 1), (3329, 2817, 520, 0.5, 1),
                                              (1100, 1000, 96, 0.0, 12)])
def test_bf16_wide_tiles_match_single_ctas(cuda, ta, tb, M, N, K, beta, batch):
    # the default BF16 path for large products (256 x 256 single-CTA tiles, all
    # of K in TMEM; at least 148 of them here) and 128 x 256 tiles run the same
    # MMA sequence per element
    A = oracle.uniform(batch * M * K, seed=31 + ta)
    B = oracle.uniform(batch * K * N, seed=32 + tb)
    Cin = oracle.uniform(batch * M * N, seed=33)
    wide = _mm(cuda, A, B, M, N, K, "tc_bf16", ta, tb, gemm=True, Cin=Cin, alpha=1.25, beta=beta, batch=batch)
    try:
        g.set_option("tc_pair", 0)
        single = _mm(cuda, A, B, M, N, K, "tc_bf16", ta, tb, gemm=True, Cin=Cin, alpha=1.25, beta=beta, batch=batch)
    finally:
        g.set_option("tc_pair", 1)
    assert np.array_equal(wide, single)
    ref = oracle.matmul(A, B, M, N, K, ta, tb, mode=oracle.F64, gemm=1, Cin=Cin, alpha=1.25, beta=beta, packed=batch)
    assert oracle.normwise_error(wide, ref) <= BUDGET["tc_bf16"]


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("rows", [128, 384, 65536])
def test_raster_group_height_does_not_change_results(cuda, engine, rows):
    # the persistent kernels visit tiles in groups of `rows` rows of C; every tile
    # is computed the same way whatever the order (batched, ragged edges, both
    # store paths: N = 700 keeps C's rows 16-byte aligned, N = 701 does not)
    M, K, P = 1100, 300, 2
    for N in (700, 701):
        A = oracle.uniform(P * M * K, seed=21)
        B = oracle.uniform(P * K * N, seed=22)
        base = _mm(cuda, A, B, M, N, K, engine, batch=P)
        g.set_option("tc_group_rows", rows)
        try:
            got = _mm(cuda, A, B, M, N, K, engine, batch=P)
        finally:
            g.set_option("tc_group_rows", 2048)
        assert np.array_equal(base, got)
        ref = oracle.matmul(A, B, M, N, K, mode=oracle.F64, packed=P)
        assert oracle.normwise_error(got, ref) <= BUDGET[engine]


@pytest.mark.parametrize("engine", ENGINES + ["tc_fp8"])
@pytest.mark.parametrize("pair", [0, 2])
def test_l2_hint_does_not_change_results(cuda, engine, pair):
    # an eviction priority on A's loads changes what stays in L2, not what is
    # loaded: single CTAs and CTA pairs, batched, ragged edges
    M, N, K, P = 700, 520, 400, 2
    A = oracle.uniform(P * M * K, seed=41)
    B = oracle.uniform(P * K * N, seed=42)
    assert g.get_option("tc_l2_hint") == 1
    try:
        g.set_option("tc_pair", pair)
        hinted = _mm(cuda, A, B, M, N, K, engine, batch=P)
        g.set_option("tc_l2_hint", 0)
        plain = _mm(cuda, A, B, M, N, K, engine, batch=P)
    finally:
        g.set_option("tc_l2_hint", 1)
        g.set_option("tc_pair", 1)
    assert np.array_equal(hinted, plain)


@pytest.mark.parametrize("engine", ENGINES + ["tc_fp8", "buffer"])
@pytest.mark.parametrize("ta,tb", [(0, 0), (1, 1), (1, 0)])
def test_host_buffer_entry_matches_device_path(cuda, engine, ta, tb):
    # M = 2300: the tensor-core engines pipeline five row blocks (the last ragged);
    # the SIMT engine takes the plain upload / run / download path
    import torch
    M, N, K = 2300, 384, 300
    A = oracle.uniform(M * K, seed=5 + ta)
    B = oracle.uniform(K * N, seed=6 + tb)
    C0 = oracle.uniform(M * N, seed=7)
    dev = _mm(cuda, A, B, M, N, K, engine, ta, tb, gemm=True, Cin=C0, alpha=0.5, beta=2.0)
    hA = torch.from_numpy(A).pin_memory()
    hB = torch.from_numpy(B).pin_memory()
    hC = torch.from_numpy(C0.copy()).pin_memory()
    g.matmul_host(hA, hB, M, N, K, hC, trans_a=ta, trans_b=tb, gemm=True, alpha=0.5, beta=2.0, engine=engine)
    torch.cuda.synchronize()
    assert g.device_faults() == 0
    assert np.array_equal(hC.numpy(), dev)


@pytest.mark.parametrize("engine,M,batch", [("buffer", 300, 2), ("tc_split3", 1100, 1), ("tc_split3", 300, 2),
                                            ("tc_bf16", 1100, 1)])
def test_host_buffer_entry_with_padded_strides(cuda, engine, M, batch):
    """Host buffers sized to their exact extent, lda > K, ldb > N, ldc > N and
    gaps between instances: the result equals the device entry point on the
    same layout, and padding columns and gaps of C keep the caller's values."""
    import torch
    N, K = 200, 150
    lda, ldb, ldc = K + 5, N + 3, N + 7
    sa, sb, sc = lda * M + 11, ldb * K + 13, ldc * M + 17
    ext = lambda st, rows, ld, inner: (batch - 1) * st + (rows - 1) * ld + inner
    a_el, b_el, c_el = ext(sa, M, lda, K), ext(sb, K, ldb, N), ext(sc, M, ldc, N)
    A = oracle.uniform(a_el, seed=31)
    B = oracle.uniform(b_el, seed=32)
    C0 = np.full(c_el, 7.25, dtype=np.float32)
    kw = dict(lda=lda, ldb=ldb, ldc=ldc, stride_a=sa, stride_b=sb, stride_c=sc)
    d = g.matmul_desc(M, N, K, engine=engine, batch=batch, **kw)
    dC = torch.from_numpy(C0.copy()).to(cuda)
    dA, dB = torch.from_numpy(A).to(cuda), torch.from_numpy(B).to(cuda)
    g.check(g.lib().gatlas_matmul_f32(ctypes.byref(d), g._ptr(dA), g._ptr(dB), g._ptr(dC), None, 0, g._stream()))
    hC = torch.from_numpy(C0.copy()).pin_memory()
    g.matmul_host(torch.from_numpy(A).pin_memory(), torch.from_numpy(B).pin_memory(), M, N, K, hC,
                  engine=engine, batch=batch, **kw)
    torch.cuda.synchronize()
    assert g.device_faults() == 0
    got, want = hC.numpy(), dC.cpu().numpy()
    assert np.array_equal(got, want)
    written = np.zeros(c_el, dtype=bool)
    for p in range(batch):
        for r in range(M):
            written[p * sc + r * ldc: p * sc + r * ldc + N] = True
    assert np.all(got[~written] == 7.25)
    for p in range(batch):
        Ap = np.stack([A[p * sa + r * lda: p * sa + r * lda + K] for r in range(M)]).ravel()
        Bp = np.stack([B[p * sb + r * ldb: p * sb + r * ldb + N] for r in range(K)]).ravel()
        Cp = np.stack([got[p * sc + r * ldc: p * sc + r * ldc + N] for r in range(M)]).ravel()
        ref = oracle.matmul(Ap, Bp, M, N, K, mode=oracle.F64)
        assert oracle.normwise_error(Cp, ref) <= (2.0 ** -7 if engine == "tc_bf16" else 8e-6)


def test_host_buffer_entry_small_and_pageable(cuda):
    import torch
    M, N, K = 100, 70, 50
    A = oracle.uniform(M * K, seed=1)
    B = oracle.uniform(K * N, seed=2)
    hC = torch.zeros(M * N)
    g.matmul_host(torch.from_numpy(A), torch.from_numpy(B), M, N, K, hC, engine="tc_split3")
    torch.cuda.synchronize()
    assert np.array_equal(hC.numpy(), _mm(cuda, A, B, M, N, K, "tc_split3"))
    with pytest.raises(ValueError):
        g.matmul_host(torch.from_numpy(A).to(cuda), torch.from_numpy(B), M, N, K, hC)
