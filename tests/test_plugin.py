"""The C++ plugin layer (KernelInterface objects) against the oracle's
restatement of the reference's parameter rules, over broad sweeps (CPU)."""
import itertools
import json
import os
import random

import pytest

from gatlas_b200.plugin import Kernel
from oracle.params import MATMUL_TYPES, Matmul, Matvec, Saxpy, journal_key

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _oracle_matmul(t):
    v, sc, vl, _, _ = MATMUL_TYPES[t]
    return Matmul(variant=v, scalar=sc, vl=vl)


@pytest.mark.parametrize("t", list(MATMUL_TYPES))
def test_matmul_rules_match_oracle(t):
    rng = random.Random(hash(t) & 0xFFFF)
    k = Kernel("matmul", t)
    o = _oracle_matmul(t)
    assert k.kernel_name() == o.kernel_name()
    assert k.total_variations() == o.total_variations()
    dims = [0, 1, 8, 48, 64, 96, 128, 640, 1024, 3520]
    for _ in range(3000):
        p = [rng.choice([0, 1, 1, 3]), rng.randint(0, 1), rng.choice(dims), rng.choice(dims),
             rng.choice(dims), rng.randint(0, 1), rng.randint(0, 1), rng.choice([0, 1, 4, 8, 9, 10, 16]),
             rng.choice([1, 4, 8, 9, 10, 16]), rng.choice([0, 1, 2, 4, 5, 8, 10, 12]),
             rng.choice([1, 2, 4, 8]), rng.randint(0, 30)]
        k.set_params(p)
        o.set_params(p)
        ok, got = k.get_params()
        assert ok == o.valid(), p
        if ok:
            assert got == o.params()
            assert k.number_flops() == o.number_flops()
            assert k.global_work_items() == o.global_work_items()
            assert k.local_work_items() == o.local_work_items()
        assert k.extra_param_detail() == o.extra_param_detail()


@pytest.mark.parametrize("t", ["float1", "float4", "double2", "floatimg"])
def test_matvec_rules_match_oracle(t):
    rng = random.Random(7)
    v, sc, vl, _, _ = MATMUL_TYPES[t]
    k = Kernel("matvec", t)
    o = Matvec(variant=v, scalar=sc, vl=vl)
    assert k.kernel_name() == o.kernel_name()
    dims = [0, 4, 64, 256, 1024, 16384, 3000]
    for _ in range(2000):
        p = [rng.choice([0, 1, 2]), rng.randint(0, 1), rng.choice(dims), rng.choice(dims),
             rng.randint(0, 1), rng.choice([0, 1, 16, 64, 65, 128, 256]), rng.choice([0, 1, 2, 4, 8, 64]),
             rng.choice([1, 2, 4]), rng.randint(0, 5)]
        k.set_params(p)
        o.set_params(p)
        ok, got = k.get_params()
        assert ok == o.valid(), p
        if ok:
            assert got == o.params()
            assert k.number_flops() == o.number_flops()
            assert k.global_work_items() == o.global_work_items()
        assert k.extra_param_detail() == o.extra_param_detail()


@pytest.mark.parametrize("t", ["float4", "double1", "floatimg"])
def test_saxpy_rules_match_oracle(t):
    rng = random.Random(11)
    v, sc, vl, _, _ = MATMUL_TYPES[t]
    k = Kernel("saxpy", t)
    o = Saxpy(variant=v, scalar=sc, vl=vl)
    for _ in range(2000):
        p = [rng.choice([0, 1, 2]), rng.choice([0, 64, 4096, 1 << 20]), rng.choice([1, 2, 4, 8, 64]),
             rng.choice([0, 1, 64, 256]), rng.choice([0, 1, 4, 16]), rng.choice([0, 1, 2, 4, 16]),
             rng.choice([0, 1, 2, 4, 8]), rng.choice([1, 2, 4]), rng.randint(0, 5)]
        k.set_params(p)
        o.set_params(p)
        ok, got = k.get_params()
        assert ok == o.valid(), p
        if ok:
            assert got == o.params()
            assert k.number_flops() == o.number_flops()
            assert k.global_work_items() == o.global_work_items()
            assert k.local_work_items() == o.local_work_items()


def test_reference_printed_points_through_plugin():
    ex = json.load(open(os.path.join(GOLDEN, "reference_examples.json")))
    for e in ex["matmul"]:
        k = Kernel("matmul", e["type"])
        k.set_params(e["params"])
        ok, p = k.get_params()
        assert ok and p == e["params"]
        assert k.extra_param_detail() == e["extra_detail"]
        if e["gflops"] is not None and e["trials"] == 1:
            assert k.number_flops() / e["usec"] / 1000 == pytest.approx(e["gflops"], rel=5e-6)
    for e in ex["journal_keys"]:
        k = Kernel("matmul", e["type"])
        assert journal_key(k.kernel_name(), e["params"]) == e["line"].split("\t")[0]


def test_tensor_core_types():
    for t, name in (("tcbf16", "matmultcbf16float4"), ("split3", "matmultcsplit3float4"),
                    ("split6", "matmultcsplit6float4"), ("fp8", "matmultcfp8float4")):
        assert Kernel("matmul", t).kernel_name() == name
    with pytest.raises(Exception):
        Kernel("matvec", "split3")
    with pytest.raises(Exception):
        Kernel("matmul", "float3")


def test_print_describes_the_cuda_instance():
    k = Kernel("matmul", "float4")
    k.set_params([1, 0, 1024, 1024, 1024, 0, 0, 16, 16, 8, 4, 3])
    text = k.print()
    assert "gemm_simt_kernel<float" in text and "GH=16" in text and "BH=8" in text
    assert "extra parameter 3 = (1 1)" in text
    assert "template __global__ void gatlas::simt::gemm_simt_kernel<float, false, false, 16, 16, 8, 4, 4, 8>" in text


def test_print_image_instance_carries_image_source():
    k = Kernel("matmul", "floatimg")
    k.set_params([1, 0, 1024, 1024, 1024, 1, 0, 16, 16, 8, 4, 0])
    text = k.print()
    assert "gemm_image_kernel<float, TA=1, TB=0" in text and "BK=32" in text
    assert "template __global__ void gatlas::img::gemm_image_kernel<float, true, false, 16, 16, 8, 4>" in text


def _nvrtc_compile(src):
    """Compiles src for sm_100a with NVRTC (no GPU needed); returns (status, log)."""
    import ctypes
    try:
        nv = ctypes.CDLL("libnvrtc.so.12")
    except OSError:
        pytest.skip("NVRTC is not installed")
    prog = ctypes.c_void_p()
    assert nv.nvrtcCreateProgram(ctypes.byref(prog), src.encode(), b"point.cu", 0, None, None) == 0
    opts = [b"--gpu-architecture=sm_100a", b"-std=c++17", b"-default-device", b"-lineinfo"]
    rc = nv.nvrtcCompileProgram(prog, len(opts), (ctypes.c_char_p * len(opts))(*opts))
    n = ctypes.c_size_t()
    nv.nvrtcGetProgramLogSize(prog, ctypes.byref(n))
    log = ctypes.create_string_buffer(n.value)
    nv.nvrtcGetProgramLog(prog, log)
    nv.nvrtcDestroyProgram(ctypes.byref(prog))
    return rc, log.value.decode(errors="replace")


@pytest.mark.parametrize("t,p", [
    ("float4", [1, 0, 640, 640, 640, 1, 0, 10, 10, 8, 4, 0]),
    ("double1", [1, 1, 640, 640, 640, 0, 1, 8, 8, 10, 1, 2]),
    ("floatimg", [1, 0, 640, 640, 640, 0, 1, 10, 10, 8, 4, 0]),
    ("floatimg", [1, 0, 768, 768, 768, 0, 0, 16, 16, 12, 4, 0]),
    ("doubleimg", [1, 0, 648, 648, 648, 1, 0, 9, 9, 4, 4, 0]),
])
def test_run_time_compiled_source_compiles(t, p):
    # the source print() shows is exactly what run-time compilation builds
    k = Kernel("matmul", t)
    k.set_params(p)
    text = k.print()
    src = text[text.index("\n\n") + 2:]
    rc, log = _nvrtc_compile(src)
    assert rc == 0, log
