"""The C-ABI library loads and exports every entry point include/*.h declares
(CPU; no compute calls)."""
import ctypes
import glob
import os
import re

import pytest

import gatlas_b200 as g

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(gatlas_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    lib = g.lib()
    names = declared_symbols()
    assert len(names) >= 15
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings_and_version():
    lib = g.lib()
    assert lib.gatlas_version() >= 100
    assert lib.gatlas_status_string(0) == b"ok"
    assert lib.gatlas_status_string(-3) == b"unsupported parameter point"


def test_argument_errors_need_no_gpu():
    lib = g.lib()
    # null descriptors and pointers are rejected before any CUDA call
    assert lib.gatlas_matmul_f32(None, None, None, None, None, 0, None) == g.ERR_INVALID
    assert "null descriptor" in g.last_error()
    assert lib.gatlas_matvec_f32(None, None, None, None, None, 0, None) == g.ERR_INVALID
    assert lib.gatlas_saxpy_f32(0, 16, ctypes.c_float(1.0), None, None, None, None) == g.ERR_INVALID
    assert lib.gatlas_saxpy_f32(7, 0, ctypes.c_float(1.0), None, None, None, None) == 0  # n == 0 is a no-op
    d = g.matmul_desc(8, 8, 8, engine=9)
    assert lib.gatlas_matmul_f32(ctypes.byref(d), ctypes.c_void_p(16), ctypes.c_void_p(16),
                                 ctypes.c_void_p(16), None, 0, None) == g.ERR_INVALID


def test_compiled_simt_points_cover_the_tuning_grid():
    # work group {8,16}^2 x blocking {4,8}^2 x vector width {1,2,4}, no transposes
    for gh in (8, 16):
        for gw in (8, 16):
            for bh in (4, 8):
                for bw in (4, 8):
                    for vl in (1, 2, 4):
                        assert g.matmul_supported("buffer", (gh, gw, bh, bw, vl)) == 1
    # other points of the reference's space are compiled at run time
    assert g.matmul_supported("buffer", (10, 10, 7, 4, 4)) == 2
    assert g.matmul_supported("buffer", (9, 9, 5, 4, 4), trans_a=True) == 0   # 45 rows not a multiple of 4
    assert g.matmul_supported("buffer", (8, 8, 4, 4, 3)) == 0


def test_workspace_queries():
    assert g.matvec_workspace_size(16384, 16384, trans_a=False) == 0
    assert g.matvec_workspace_size(16384, 16384, trans_a=True) > 0
    assert g.matmul_workspace_size(1024, 1024, 1024, "buffer") == 0


def test_options_round_trip_without_a_device():
    import gatlas_b200 as g
    assert g.get_option("tc_pair") == 1
    g.set_option("tc_pair", 0)
    try:
        assert g.get_option("tc_pair") == 0
    finally:
        g.set_option("tc_pair", 1)
    with pytest.raises(g.GatlasError, match="unknown option"):
        g.set_option("no_such_option", 1)
    with pytest.raises(g.GatlasError, match="0, 1 or 2"):
        g.set_option("tc_pair", 3)
    assert g.get_option("tc_l2_hint") == 1
    with pytest.raises(g.GatlasError, match="0 or 1"):
        g.set_option("tc_l2_hint", 2)
    assert g.get_option("grouped_pair") == 0
    g.set_option("grouped_pair", 1)
    try:
        assert g.get_option("grouped_pair") == 1
    finally:
        g.set_option("grouped_pair", 0)
    with pytest.raises(g.GatlasError, match="single CTAs"):
        g.set_option("grouped_pair", 2)
    assert g.get_option("tc_group_rows") == 2048
    g.set_option("tc_group_rows", 384)
    try:
        assert g.get_option("tc_group_rows") == 384
    finally:
        g.set_option("tc_group_rows", 2048)
    for bad in (0, 100, 129, 65536 + 128):
        with pytest.raises(g.GatlasError, match="multiple of 128"):
            g.set_option("tc_group_rows", bad)
    assert g.get_option("host_block_rows") == 512
    g.set_option("host_block_rows", 1024)
    try:
        assert g.get_option("host_block_rows") == 1024
    finally:
        g.set_option("host_block_rows", 512)
    for bad in (0, 128, 300):
        with pytest.raises(g.GatlasError, match="multiple of 256"):
            g.set_option("host_block_rows", bad)


@pytest.mark.parametrize("M,N", [(65536, 65536), (131072, 8192), (32768, 262144)])
def test_matvec_workspace_query_covers_the_image_engine(M, N):
    """The allocation-free GEMV states the scratch its column-major TMA path
    needs when that is more than its static array, before any CUDA call; the
    workspace query must never report less for the same problem.  The operand
    pointers are NULL: the size check comes first, and any path past it stops
    at the null-pointer check, so no kernel can launch."""
    lib = g.lib()
    d = g.matvec_desc(M, N, trans_a=True, engine="image")
    assert lib.gatlas_matvec_f32_noalloc(ctypes.byref(d), None, None, None, None) == g.ERR_INVALID
    need = int(re.search(r"needs (\d+) bytes", g.last_error()).group(1))
    assert need > 1 << 20
    assert g.matvec_workspace_size(M, N, trans_a=True) >= need


@pytest.mark.parametrize("engine", ["tc_bf16", "tc_split3", "tc_split6", "tc_fp8"])
@pytest.mark.parametrize("M,N,K,ta,tb,batch", [(1000, 700, 333, 0, 0, 1), (4096, 4096, 4096, 1, 1, 1),
                                               (129, 257, 1000, 0, 1, 3), (16, 16, 16, 1, 0, 65535)])
def test_tc_prepare_asks_for_exactly_the_queried_workspace(engine, M, N, K, ta, tb, batch, no_cuda_device):
    """tc_prepare rejects a workspace one byte short of gatlas_matmul_workspace_size
    with the size it needs, which is the query's (before any device work)."""
    need = g.matmul_workspace_size(M, N, K, engine, ta, tb, batch)
    assert need > 0
    d = g.matmul_desc(M, N, K, ta, tb, engine=engine, batch=batch)
    p = ctypes.c_void_p(1 << 20)
    rc = g.lib().gatlas_matmul_tc_prepare(ctypes.byref(d), p, p, p, need - 1, None)
    assert rc == g.ERR_INVALID
    assert int(re.search(r"workspace \d+ < (\d+) bytes", g.last_error()).group(1)) == need
    rc = g.lib().gatlas_matmul_tc_prepare(ctypes.byref(d), p, p, ctypes.c_void_p((1 << 20) + 512), need, None)
    assert rc == g.ERR_INVALID and "1024-byte aligned" in g.last_error()
