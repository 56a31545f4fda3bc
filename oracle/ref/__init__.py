"""The reference's own generated kernels, run on the host CPU.

TEST INFRASTRUCTURE ONLY: tests/ use these kernels to pin the oracle's
restatement against the reference itself, and bench.py's reference arm and
cpu_baseline leg time them.  The product (gatlas_b200) never imports this.

oracle/ref/Makefile builds oracle/_ref/librefk.so from the reference's
sources (where they are present); the built library and its manifest
oracle/_ref/kernels.json travel with the repository copy, so machines
without the reference's sources run the prebuilt kernels.
"""

from __future__ import annotations

import ctypes
import json
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_OUT = os.path.join(os.path.dirname(_HERE), "_ref")
LIB_PATH = os.path.join(_OUT, "librefk.so")
MANIFEST = os.path.join(_OUT, "kernels.json")
REF_SRC = os.environ.get("GATLAS_REF_SRC", "/root/reference")

_lib = None
_kernels = None


class RefkArgs(ctypes.Structure):
    _fields_ = [("A", ctypes.c_void_p), ("B", ctypes.c_void_p), ("C", ctypes.c_void_p),
                ("alpha", ctypes.c_double), ("beta", ctypes.c_double),
                ("group_begin", ctypes.c_size_t * 2), ("group_end", ctypes.c_size_t * 2),
                ("threads", ctypes.c_int)]


def sources_present() -> bool:
    return os.path.isdir(REF_SRC) and os.path.exists(os.path.join(REF_SRC, "KernelMatmulBuffer.hpp"))


def available() -> bool:
    return os.path.exists(LIB_PATH) and os.path.exists(MANIFEST)


def build() -> None:
    """Builds (or refreshes) oracle/_ref from the reference's sources."""
    if not sources_present():
        raise RuntimeError(f"reference sources not found at {REF_SRC}")
    subprocess.run(["make", "-s", "-C", _HERE, f"REF_SRC={REF_SRC}", "-j", str(os.cpu_count() or 4)],
                   check=True)


def lib() -> ctypes.CDLL:
    global _lib, _kernels
    if _lib is None:
        if not available():
            build()
        _lib = ctypes.CDLL(LIB_PATH)
        with open(MANIFEST) as f:
            _kernels = {k["id"]: k for k in json.load(f)}
    return _lib


def kernels() -> dict:
    lib()
    return _kernels


def kernel(kid: str) -> dict:
    return kernels()[kid]


def groups(kid: str) -> tuple[int, int]:
    k = kernel(kid)
    return k["global"][0] // k["local"][0], k["global"][1] // k["local"][1]


def run(kid: str, A: np.ndarray, B: np.ndarray, C: np.ndarray, alpha: float = 1.0, beta: float = 0.0,
        fused: bool = True, group_begin=(0, 0), group_end=(0, 0), threads: int = 0) -> np.ndarray:
    """Runs kernel `kid` on flat row-major host arrays in the reference's
    layouts (matmul A, B, C; matvec A, x, y; saxpy X, Y, Z).  C is written in
    place (and read first by GEMM/GEMV kernels); returns C."""
    L = lib()
    k = _kernels[kid]
    dt = np.float64 if k["scalar"] == "double" else np.float32
    for a in (A, B, C):
        if a.dtype != dt or not a.flags.c_contiguous:
            raise ValueError(f"{kid}: operands must be contiguous {np.dtype(dt).name} arrays")
    fn = getattr(L, f"refk_{kid}_{'fma' if fused else 'sep'}")
    fn.argtypes = [ctypes.POINTER(RefkArgs)]
    fn.restype = ctypes.c_int
    args = RefkArgs(A.ctypes.data, B.ctypes.data, C.ctypes.data, alpha, beta,
                    (ctypes.c_size_t * 2)(*group_begin), (ctypes.c_size_t * 2)(*group_end), threads)
    rc = fn(ctypes.byref(args))
    if rc != 0:
        raise RuntimeError(f"{kid}: work-group runner failed ({rc})")
    return C
