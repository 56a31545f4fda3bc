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


def test_fma_within_normwise_4ku_of_f64():
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


# ---- FP8 E4M3 block quantisation (operand format of the FP8 tensor-core engine) ----

def _e4m3_by_search(x):
    """Independent restatement: nearest finite E4M3 value, ties to the even
    code, saturating at 448."""
    vals = np.array([oracle.e4m3_decode(np.array([c], np.uint8))[0] for c in range(127)], np.float64)
    out = np.empty(x.size, np.uint8)
    for i, v in enumerate(x.astype(np.float64)):
        a = min(abs(v), 448.0)
        d = np.abs(vals - a)
        best = np.flatnonzero(d == d.min())
        c = best[0] if len(best) == 1 else [b for b in best if b % 2 == 0][0]
        out[i] = c | (0x80 if np.signbit(v) else 0)
    return out


def test_e4m3_code_table_and_round_trip():
    vals = oracle.e4m3_decode(np.arange(256, dtype=np.uint8))
    assert vals[0x01] == 2.0 ** -9 and vals[0x08] == 2.0 ** -6 and vals[0x7E] == 448.0
    assert np.isnan(vals[0x7F]) and np.isnan(vals[0xFF]) and vals[0xFE] == -448.0
    finite = [c for c in range(256) if c not in (0x7F, 0xFF)]
    assert np.array_equal(oracle.e4m3_encode(vals[finite]), np.array(finite, np.uint8))


def test_e4m3_rounding_matches_nearest_search():
    rng = np.random.default_rng(5)
    pos = oracle.e4m3_decode(np.arange(127, dtype=np.uint8)).astype(np.float64)
    mids = (pos[1:] + pos[:-1]) / 2                        # exact ties
    x = np.concatenate([
        mids, np.nextafter(mids, 0), np.nextafter(mids, 1e9),
        rng.uniform(-1, 1, 2000) * 2.0 ** rng.integers(-12, 10, 2000),
        [0.0, -0.0, 2.0 ** -10, 3 * 2.0 ** -11, 447.9, 448.0, 463.9, 464.0, 1e6, -1e6, 2.0 ** -20],
    ]).astype(np.float32)
    x = np.concatenate([x, -x])
    assert np.array_equal(oracle.e4m3_encode(x), _e4m3_by_search(x))


@pytest.mark.parametrize("transposed", [0, 1])
def test_fp8_block_quantisation_properties(transposed):
    rows, K = 200, 300
    src = oracle.uniform(rows * K, seed=9) * np.float32(3.0)
    src[:5] = 0.0
    codes, scales = oracle.quant_fp8(src, rows, K, transposed)
    assert codes.shape == (1, rows, 304) and scales.shape == (1, 2, 3)
    assert not codes[0, :, K:].any()                        # zero padding up to Kp
    view = src.reshape(K, rows).T if transposed else src.reshape(rows, K)
    deq = oracle.e4m3_decode(codes[0, :, :K].ravel()).reshape(rows, K).astype(np.float64)
    deq *= np.repeat(np.repeat(scales[0], 128, 0), 128, 1)[:rows, :K]
    for rb in range(2):
        for kb in range(3):
            blk = view[rb * 128:(rb + 1) * 128, kb * 128:(kb + 1) * 128]
            amax, sc = float(np.abs(blk).max()), float(scales[0, rb, kb])
            assert sc == 2.0 ** np.ceil(np.log2(amax / 448.0))   # smallest power of two with amax/s <= 448
            cb = codes[0, rb * 128:(rb + 1) * 128, kb * 128:min((kb + 1) * 128, K)]
            assert oracle.e4m3_decode(np.array([(cb & 0x7F).max()], np.uint8))[0] > 224  # top binade used
    # relative error of every element at most half an E4M3 ulp (2^-4) above the subnormal range
    big = np.abs(view) >= np.repeat(np.repeat(scales[0], 128, 0), 128, 1)[:rows, :K] * 2.0 ** -6
    assert np.all(np.abs(deq - view)[big] <= 2.0 ** -4 * np.abs(view)[big])


def test_fp8_dequant_product_of_exact_codes():
    # operands that quantise exactly (E4M3 values with block max 448 -> scale 1):
    # the dequantised product equals the FP64 product of the operands
    M, N, K = 64, 48, 160
    rng = np.random.default_rng(2)
    vals = oracle.e4m3_decode(np.arange(127, dtype=np.uint8))
    A = rng.choice(vals, M * K).astype(np.float32) * rng.choice([-1, 1], M * K).astype(np.float32)
    B = rng.choice(vals, K * N).astype(np.float32)
    A[0], B[0] = 448.0, 448.0
    A[K * 1 + 130], B[130 * N] = 448.0, 448.0               # second K block of both
    qa, sa = oracle.quant_fp8(A, M, K, 0)
    qb, sb = oracle.quant_fp8(B, N, K, 1)                   # B stored K x N is transposed for N x K
    assert np.all(sa == 1.0) and np.all(sb == 1.0)
    C = oracle.matmul_fp8_dequant(qa, sa, qb, sb, M, N, K)
    ref = A.astype(np.float64).reshape(M, K) @ B.astype(np.float64).reshape(K, N)
    assert np.array_equal(C.reshape(M, N), ref)


def test_fp8_power_of_two_operands_quantise_exactly():
    # sign * 2^e with e in [-8, 8]: the block maximum 2^8 gives scale 1 and every
    # value is an E4M3 code (2^-8 and 2^-7 as subnormals)
    A = oracle.pow2(256 * 256, seed=3)
    codes, scales = oracle.quant_fp8(A, 256, 256, 0)
    assert np.all(scales == 1.0)
    assert np.array_equal(oracle.e4m3_decode(codes.ravel()), A)
