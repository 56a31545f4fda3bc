"""Regenerates the golden fixtures in tests/golden/.

  python tests/golden/make_golden.py

* drand48_default.json: the first values of glibc's drand48() in a fresh
  process that never seeds it -- the stream the reference's posrand/fillrand
  draw from (OCLAppUtil.hpp:28-39).  Produced by calling libc directly, not
  the oracle, so it pins the oracle's reset-to-default-state logic.
* oracle_small.npz: small seeded cases (inputs and ORACLE_FMA / FP64 outputs)
  that the GPU tests compare against; produced by the oracle.

reference_examples.json is transcribed by hand from the reference's
documentation and is not regenerated here.
"""

from __future__ import annotations

import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402

_DRAND_SNIPPET = (
    "import ctypes, json\n"
    "libc = ctypes.CDLL('libc.so.6')\n"
    "libc.drand48.restype = ctypes.c_double\n"
    "print(json.dumps([libc.drand48() for _ in range(64)]))\n"
)


def drand48_fixture() -> None:
    out = subprocess.run([sys.executable, "-c", _DRAND_SNIPPET], check=True,
                         capture_output=True, text=True).stdout
    vals = json.loads(out)
    with open(os.path.join(HERE, "drand48_default.json"), "w") as f:
        json.dump({"_source": "glibc drand48() in a fresh process, never seeded",
                   "values": [float.hex(v) for v in vals]}, f, indent=1)


def small_fixture() -> None:
    arrays = {}
    # matmul: every layout, pure and general
    M, N, K = 40, 56, 48
    for ta in (0, 1):
        for tb in (0, 1):
            A = oracle.uniform(M * K, seed=11 + 2 * ta + tb)
            B = oracle.uniform(K * N, seed=21 + 2 * ta + tb)
            Cin = oracle.uniform(M * N, seed=31)
            tag = f"mm_t{ta}{tb}"
            arrays[f"{tag}_A"] = A
            arrays[f"{tag}_B"] = B
            arrays[f"{tag}_Cin"] = Cin
            arrays[f"{tag}_fma"] = oracle.matmul(A, B, M, N, K, ta, tb, mode=oracle.FMA)
            arrays[f"{tag}_gemm_fma"] = oracle.matmul(A, B, M, N, K, ta, tb, mode=oracle.FMA,
                                                      gemm=1, Cin=Cin, alpha=0.75, beta=-1.25)
            arrays[f"{tag}_f64"] = oracle.matmul(A, B, M, N, K, ta, tb, mode=oracle.F64)
    arrays["mm_dims"] = np.array([M, N, K])
    # matvec: both layouts
    M, N = 96, 80
    for ta in (0, 1):
        A = oracle.uniform(M * N, seed=41 + ta)
        x = oracle.uniform(N, seed=51 + ta)
        yin = oracle.uniform(M, seed=61)
        arrays[f"mv_t{ta}_A"] = A
        arrays[f"mv_t{ta}_x"] = x
        arrays[f"mv_t{ta}_yin"] = yin
        arrays[f"mv_t{ta}_f64"] = oracle.matvec(A, x, M, N, ta, mode=oracle.F64)
        arrays[f"mv_t{ta}_gemv_f64"] = oracle.matvec(A, x, M, N, ta, mode=oracle.F64, gemv=1,
                                                     cin=yin, alpha=0.5, beta=2.0)
    arrays["mv_dims"] = np.array([M, N])
    # saxpy
    n = 1001
    x = oracle.uniform(n, seed=71)
    y = oracle.uniform(n, seed=72)
    arrays["sx_x"] = x
    arrays["sx_y"] = y
    arrays["sx_fma"] = oracle.saxpy(0.5, x, y, mode=oracle.FMA)
    arrays["sx_refhost"] = oracle.saxpy(0.5, x, y, mode=oracle.REFHOST)
    np.savez_compressed(os.path.join(HERE, "oracle_small.npz"), **arrays)


if __name__ == "__main__":
    drand48_fixture()
    small_fixture()
    print("golden fixtures written to", HERE)
