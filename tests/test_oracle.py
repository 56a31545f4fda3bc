"""The oracle against the reference's known answers and golden vectors (CPU)."""
import json
import os

import numpy as np
import pytest

import oracle

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_drand48_stream_matches_unseeded_glibc():
    vals = [float.fromhex(h) for h in json.load(open(os.path.join(GOLDEN, "drand48_default.json")))["values"]]
    oracle.drand48_reset()
    got = [oracle.lib().oracle_drand48() for _ in range(len(vals))]
    assert got == vals


def test_posrand_rounds_to_float_and_skips_zero():
    # posrand<float> = (float)drand48(), retried while zero (OCLAppUtil.hpp:28-33)
    vals = [float.fromhex(h) for h in json.load(open(os.path.join(GOLDEN, "drand48_default.json")))["values"]]
    oracle.drand48_reset()
    f = oracle.fillrand(16, np.float32)
    assert np.array_equal(f, np.array(vals[:16], dtype=np.float32))
    oracle.drand48_reset()
    d = oracle.fillrand(16, np.float64)
    assert np.array_equal(d, np.array(vals[:16]))


@pytest.mark.parametrize("mode", [oracle.REFHOST, oracle.FMA])
@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("packed", [1, 3])
def test_matmul_known_answer(mode, ta, tb, packed):
    # A = B = 1  =>  C == K exactly (KernelMatmulBuffer.hpp:77-79)
    M, N, K = 24, 40, 56
    A = np.ones(packed * M * K, np.float32)
    B = np.ones(packed * K * N, np.float32)
    C = oracle.matmul(A, B, M, N, K, ta, tb, mode=mode, packed=packed)
    assert oracle.check_pattern(C, float(K))
    Cd = oracle.matmul(A.astype(np.float64), B.astype(np.float64), M, N, K, ta, tb, mode=mode,
                       packed=packed, dtype=np.float64)
    assert oracle.check_pattern(Cd, float(K))


@pytest.mark.parametrize("mode", [oracle.REFHOST, oracle.FMA])
@pytest.mark.parametrize("ta", [0, 1])
def test_matvec_known_answer(mode, ta):
    M, N = 48, 72
    c = oracle.matvec(np.ones(2 * M * N, np.float32), np.ones(2 * N, np.float32), M, N, ta,
                      mode=mode, packed=2)
    assert oracle.check_pattern(c, float(N))


def test_saxpy_known_answer():
    z = oracle.saxpy(1.0, np.ones(1000, np.float32), np.ones(1000, np.float32), mode=oracle.REFHOST)
    assert oracle.check_pattern(z, 2.0)


def test_gemm_test_pattern_with_alpha_beta_one():
    # the reference's GEMM test pattern: alpha = beta = 1, C cleared to 0 => C == K
    M = N = K = 32
    C = oracle.matmul(np.ones(M * K, np.float32), np.ones(K * N, np.float32), M, N, K,
                      mode=oracle.FMA, gemm=1, Cin=np.zeros(M * N, np.float32), alpha=1.0, beta=1.0)
    assert oracle.check_pattern(C, float(K))


def test_modes_agree_on_exact_products():
    # sign*2^e inputs: every product is exact, so a fused multiply-add rounds
    # exactly like a separate product and sum: REFHOST == FMA bit for bit
    M, N, K = 16, 24, 64
    A = oracle.pow2(M * K, seed=1)
    B = oracle.pow2(K * N, seed=2)
    r = oracle.matmul(A, B, M, N, K, mode=oracle.REFHOST)
    f = oracle.matmul(A, B, M, N, K, mode=oracle.FMA)
    assert np.array_equal(r, f)


def test_refhost_is_unfused():
    # one case where fma and separate rounding differ: a*b + c with an inexact product
    a = np.array([1.0 + 2.0 ** -12], np.float32)
    x = np.array([1.0 + 2.0 ** -12], np.float32)
    y = np.array([-1.0], np.float32)
    fused = oracle.saxpy(float(a[0]), x, y, mode=oracle.FMA)
    unfused = oracle.saxpy(float(a[0]), x, y, mode=oracle.REFHOST)
    assert fused[0] != unfused[0]
    assert fused[0] == np.float32(np.float64(a[0]) * np.float64(x[0]) - 1.0)


def test_tiled_port_equals_fma_chain():
    M, N, K = 70, 45, 33
    for ta in (0, 1):
        for tb in (0, 1):
            A = oracle.uniform(M * K, seed=3)
            B = oracle.uniform(K * N, seed=4)
            ref = oracle.matmul(A, B, M, N, K, ta, tb, mode=oracle.FMA)
            til = oracle.matmul_tiled(A, B, M, N, K, ta, tb, tile_m=32, tile_n=16)
            assert np.array_equal(ref, til)


def test_fma_within_north_star_tolerance_of_f64():
    M, N, K = 64, 64, 512
    A = oracle.uniform(M * K, seed=5)
    B = oracle.uniform(K * N, seed=6)
    f = oracle.matmul(A, B, M, N, K, mode=oracle.FMA)
    d = oracle.matmul(A, B, M, N, K, mode=oracle.F64)
    assert oracle.normwise_error(f, d) <= 4 * K * 2.0 ** -24


def test_paranoid_criterion():
    a = np.zeros(100, np.float32)
    b = a.copy()
    assert oracle.paranoid_ok(a, b)
    b[3] = 0.02  # absdiff 0.02 >= 1/100
    assert not oracle.paranoid_ok(a, b)


def test_uniform_stream_properties():
    u = oracle.uniform(1 << 16, seed=9)
    assert u.min() >= -1.0 and u.max() < 1.0
    assert abs(float(u.mean())) < 0.02
    # 24 random bits: every value is a multiple of 2^-23
    assert np.all(np.ldexp(u.astype(np.float64), 23) == np.round(np.ldexp(u.astype(np.float64), 23)))
    p = oracle.pow2(4096, seed=9)
    e = np.log2(np.abs(p.astype(np.float64)))
    assert np.all(e == np.round(e)) and e.min() == -8 and e.max() == 8
