"""Python access to the oracle (oracle.c) through ctypes.

TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline legs use it as the checker or the timed CPU baseline.  The
product (gatlas_b200) never imports it.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

REFHOST, FMA, F64 = 0, 1, 2


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        c_sz, c_int, c_u64 = ctypes.c_size_t, ctypes.c_int, ctypes.c_uint64
        vp = ctypes.c_void_p
        L.oracle_drand48.restype = ctypes.c_double
        L.oracle_posrand_f32.restype = ctypes.c_float
        L.oracle_posrand_f64.restype = ctypes.c_double
        L.oracle_fillrand_f32.argtypes = [vp, c_sz]
        L.oracle_fillrand_f64.argtypes = [vp, c_sz]
        L.oracle_splitmix64.argtypes = [c_u64]
        L.oracle_splitmix64.restype = c_u64
        for n in ("oracle_fill_uniform_f32", "oracle_fill_uniform_f64", "oracle_fill_pow2_f32"):
            getattr(L, n).argtypes = [vp, c_sz, c_u64, c_u64]
        L.oracle_matmul_f32.argtypes = [c_int, c_sz, c_int, c_sz, c_sz, c_sz, c_int, c_int,
                                        vp, vp, vp, ctypes.c_float, ctypes.c_float, vp, c_int]
        L.oracle_matmul_f32_acc64.argtypes = [c_sz, c_int, c_sz, c_sz, c_sz, c_int, c_int,
                                              vp, vp, vp, ctypes.c_double, ctypes.c_double,
                                              vp, c_int]
        L.oracle_matmul_f64.argtypes = [c_int, c_sz, c_int, c_sz, c_sz, c_sz, c_int, c_int,
                                        vp, vp, vp, ctypes.c_double, ctypes.c_double, vp, c_int]
        L.oracle_matmul_tiled_f32.argtypes = [c_sz, c_sz, c_sz, c_int, c_int, vp, vp, vp,
                                              c_sz, c_sz, c_sz, c_sz, c_int]
        L.oracle_matvec_f32.argtypes = [c_int, c_sz, c_int, c_sz, c_sz, c_int, vp, vp, vp,
                                        ctypes.c_float, ctypes.c_float, vp, c_int]
        L.oracle_matvec_f32_acc64.argtypes = [c_sz, c_int, c_sz, c_sz, c_int, vp, vp, vp,
                                              ctypes.c_double, ctypes.c_double, vp, c_int]
        L.oracle_matvec_f64.argtypes = [c_int, c_sz, c_int, c_sz, c_sz, c_int, vp, vp, vp,
                                        ctypes.c_double, ctypes.c_double, vp, c_int]
        L.oracle_saxpy_f32.argtypes = [c_int, c_sz, ctypes.c_float, vp, vp, vp, c_int]
        L.oracle_saxpy_f64.argtypes = [c_int, c_sz, ctypes.c_double, vp, vp, vp, c_int]
        L.oracle_absdiff_f32.argtypes = [vp, vp, c_sz]
        L.oracle_absdiff_f32.restype = ctypes.c_longdouble
        L.oracle_absdiff_f64.argtypes = [vp, vp, c_sz]
        L.oracle_absdiff_f64.restype = ctypes.c_longdouble
        L.oracle_check_pattern_f32.argtypes = [vp, c_sz, ctypes.c_float]
        L.oracle_check_pattern_f64.argtypes = [vp, c_sz, ctypes.c_double]
        L.oracle_max_threads.restype = c_int
        L.oracle_e4m3_encode_n.argtypes = [vp, vp, c_sz]
        L.oracle_e4m3_decode_n.argtypes = [vp, vp, c_sz]
        L.oracle_quant_fp8.argtypes = [c_sz, c_sz, c_sz, c_sz, c_int, c_sz, c_sz, vp, vp, vp]
        L.oracle_matmul_fp8_dequant.argtypes = [c_sz, c_int, c_sz, c_sz, c_sz, c_sz, vp, vp, vp, vp,
                                                ctypes.c_double, ctypes.c_double, vp, vp]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


# ---- random streams --------------------------------------------------------

def drand48_reset() -> None:
    lib().oracle_drand48_reset()


def fillrand(n: int, dtype=np.float32) -> np.ndarray:
    out = np.empty(n, dtype=dtype)
    if dtype == np.float32:
        lib().oracle_fillrand_f32(_p(out), n)
    else:
        lib().oracle_fillrand_f64(_p(out), n)
    return out


def uniform(n: int, seed: int, offset: int = 0, dtype=np.float32) -> np.ndarray:
    out = np.empty(n, dtype=dtype)
    fn = lib().oracle_fill_uniform_f32 if dtype == np.float32 else lib().oracle_fill_uniform_f64
    fn(_p(out), n, seed, offset)
    return out


def pow2(n: int, seed: int, offset: int = 0) -> np.ndarray:
    out = np.empty(n, dtype=np.float32)
    lib().oracle_fill_pow2_f32(_p(out), n, seed, offset)
    return out


# ---- ops ---------------------------------------------------------------------

def matmul(A, B, M, N, K, tA=0, tB=0, mode=FMA, gemm=0, Cin=None, alpha=1.0, beta=0.0,
           packed=1, dtype=np.float32, threads=0):
    """Returns C (packed*M*N,) for flat A (packed*M*K) and B (packed*K*N)."""
    A = _c(A, dtype).ravel()
    B = _c(B, dtype).ravel()
    Ci = None if Cin is None else _c(Cin, dtype).ravel()
    if gemm and Ci is None:
        Ci = np.zeros(packed * M * N, dtype=dtype)
    if mode == F64:
        out = np.empty(packed * M * N, dtype=np.float64)
        assert dtype == np.float32
        lib().oracle_matmul_f32_acc64(packed, gemm, M, N, K, tA, tB, _p(A), _p(B), _p(Ci),
                                      alpha, beta, _p(out), threads)
        return out
    out = np.empty(packed * M * N, dtype=dtype)
    fn = lib().oracle_matmul_f32 if dtype == np.float32 else lib().oracle_matmul_f64
    rc = fn(mode, packed, gemm, M, N, K, tA, tB, _p(A), _p(B), _p(Ci), alpha, beta, _p(out),
            threads)
    assert rc == 0
    return out


def matmul_tiled(A, B, M, N, K, tA=0, tB=0, tile_m=128, tile_n=64, row_begin=0,
                 row_end=None, threads=0):
    A = _c(A, np.float32).ravel()
    B = _c(B, np.float32).ravel()
    out = np.zeros(M * N, dtype=np.float32)
    row_end = M if row_end is None else row_end
    rc = lib().oracle_matmul_tiled_f32(M, N, K, tA, tB, _p(A), _p(B), _p(out), tile_m, tile_n,
                                       row_begin, row_end, threads)
    assert rc == 0
    return out


def matvec(A, b, M, N, tA=0, mode=FMA, gemv=0, cin=None, alpha=1.0, beta=0.0, packed=1,
           dtype=np.float32, threads=0):
    A = _c(A, dtype).ravel()
    b = _c(b, dtype).ravel()
    ci = None if cin is None else _c(cin, dtype).ravel()
    if gemv and ci is None:
        ci = np.zeros(packed * M, dtype=dtype)
    if mode == F64:
        out = np.empty(packed * M, dtype=np.float64)
        assert dtype == np.float32
        lib().oracle_matvec_f32_acc64(packed, gemv, M, N, tA, _p(A), _p(b), _p(ci), alpha, beta,
                                      _p(out), threads)
        return out
    out = np.empty(packed * M, dtype=dtype)
    fn = lib().oracle_matvec_f32 if dtype == np.float32 else lib().oracle_matvec_f64
    rc = fn(mode, packed, gemv, M, N, tA, _p(A), _p(b), _p(ci), alpha, beta, _p(out), threads)
    assert rc == 0
    return out


def saxpy(alpha, x, y, mode=FMA, dtype=np.float32, threads=0):
    x = _c(x, dtype).ravel()
    y = _c(y, dtype).ravel()
    out = np.empty_like(x)
    fn = lib().oracle_saxpy_f32 if dtype == np.float32 else lib().oracle_saxpy_f64
    rc = fn(mode, x.size, alpha, _p(x), _p(y), _p(out), threads)
    assert rc == 0
    return out


def absdiff(a, b) -> float:
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b, dtype=a.dtype)
    fn = lib().oracle_absdiff_f32 if a.dtype == np.float32 else lib().oracle_absdiff_f64
    return float(fn(_p(a), _p(b), a.size))


def paranoid_ok(out, ref) -> bool:
    """The reference's paranoid criterion: absdiff < 1/length
    (OCLAppUtil.hpp:212-264)."""
    return absdiff(out, ref) < 1.0 / np.asarray(out).size


def check_pattern(a, value) -> bool:
    a = np.ascontiguousarray(a)
    fn = lib().oracle_check_pattern_f32 if a.dtype == np.float32 else lib().oracle_check_pattern_f64
    return bool(fn(_p(a), a.size, value))


def max_threads() -> int:
    return int(lib().oracle_max_threads())


def normwise_error(C, Cref, A=None, B=None) -> float:
    """||C - Cref||_F / ||Cref||_F (or / (||A||_F ||B||_F) when A, B given)."""
    C = np.asarray(C, dtype=np.float64)
    Cref = np.asarray(Cref, dtype=np.float64)
    num = np.linalg.norm((C - Cref).ravel())
    if A is not None and B is not None:
        den = np.linalg.norm(np.asarray(A, np.float64).ravel()) * \
            np.linalg.norm(np.asarray(B, np.float64).ravel())
    else:
        den = np.linalg.norm(Cref.ravel())
    return float(num / den) if den else float(num)


# ---- FP8 E4M3 block quantisation --------------------------------------------

FP8_BLOCK = 128


def e4m3_encode(x) -> np.ndarray:
    x = _c(x, np.float32).ravel()
    out = np.empty(x.size, dtype=np.uint8)
    lib().oracle_e4m3_encode_n(_p(x), _p(out), x.size)
    return out


def e4m3_decode(c) -> np.ndarray:
    c = _c(c, np.uint8).ravel()
    out = np.empty(c.size, dtype=np.float32)
    lib().oracle_e4m3_decode_n(_p(c), _p(out), c.size)
    return out


def fp8_kp(K: int) -> int:
    """Row pitch (in codes) of the K-major FP8 operand: K rounded up to 16."""
    return (max(K, 1) + 15) // 16 * 16


def quant_fp8(src, rows: int, K: int, transposed: int, ld: int | None = None, batch: int = 1,
              src_stride: int | None = None):
    """Block quantisation of one operand viewed as rows x K (element (r,k) at
    src[r*ld + k], or src[k*ld + r] when transposed).  Returns (codes
    [batch, rows, Kp] uint8, scales [batch, rblocks, kblocks] float32)."""
    src = _c(src, np.float32).ravel()
    ld = ld if ld is not None else (rows if transposed else K)
    src_stride = src_stride if src_stride is not None else rows * K
    Kp = fp8_kp(K)
    rb, kb = -(-rows // FP8_BLOCK), -(-max(K, 1) // FP8_BLOCK)
    codes = np.zeros((batch, rows, Kp), dtype=np.uint8)
    scales = np.zeros((batch, rb, kb), dtype=np.float32)
    assert lib().oracle_quant_fp8(batch, rows, K, Kp, transposed, ld, src_stride, _p(src), _p(codes),
                                  _p(scales)) == 0
    return codes, scales


def matmul_fp8_dequant(qa, sa, qb, sb, M: int, N: int, K: int, batch: int = 1, gemm: int = 0,
                       alpha: float = 1.0, beta: float = 0.0, Cin=None) -> np.ndarray:
    """FP64 product of the dequantised operands (codes K-major: A as M x Kp, B as N x Kp)."""
    qa, qb = _c(qa, np.uint8), _c(qb, np.uint8)
    sa, sb = _c(sa, np.float32), _c(sb, np.float32)
    Ci = None if Cin is None else _c(Cin, np.float32).ravel()
    if gemm and Ci is None:
        Ci = np.zeros(batch * M * N, dtype=np.float32)
    out = np.empty(batch * M * N, dtype=np.float64)
    lib().oracle_matmul_fp8_dequant(batch, gemm, M, N, K, fp8_kp(K), _p(qa), _p(sa), _p(qb), _p(sb),
                                    alpha, beta, _p(Ci), _p(out))
    return out
