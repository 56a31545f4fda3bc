"""Grouped GEMM host logic on CPU: size buckets, the tuned tile table, the
packed workspace layout and argument validation (all before any device work)."""
import numpy as np
import pytest

import gatlas_b200 as g


def test_buckets_by_n():
    assert [g.grouped_bucket(16, n, 16) for n in (1, 64, 65, 128, 129, 256, 257, 4096)] == [0, 0, 1, 1, 2, 2, 3, 3]


def test_tile_table_round_trip_and_validation():
    old, other = g.grouped_tile_table("tc_bf16"), g.grouped_tile_table("tc_split3")
    try:
        assert g.grouped_tile_table("tc_bf16", [128, 128, 128, 256]) == [128, 128, 128, 256]
        assert g.grouped_tile_table("tc_split3") == other      # one table per engine
        with pytest.raises(g.GatlasError):
            g.grouped_tile_table("tc_bf16", [96, 128, 256, 256])
        with pytest.raises(g.GatlasError):
            g.grouped_tile_table("tc_split6", [64, 128, 256, 256])
    finally:
        g.grouped_tile_table("tc_bf16", old)


def _packed_bytes(m, n, k, bn, np_):
    r = lambda x: (x + 1023) // 1024 * 1024
    if m == 0 or n == 0:
        return 0
    # tiles of 128-byte K slices (64 BF16 elements) per row
    mt, nt, kt = -(-m // 128), -(-n // bn), -(-k // 64)
    return np_ * (r(mt * kt * 128 * 128) + r(nt * kt * bn * 128))


@pytest.mark.parametrize("engine,np_", [("tc_bf16", 1), ("tc_split3", 2)])
def test_workspace_is_the_sum_of_packed_tiles(engine, np_):
    rng = np.random.default_rng(1)
    inst = []
    for _ in range(40):
        m, n, k = (int(x) for x in rng.integers(0, 700, 3))
        inst.append(dict(m=m, n=n, k=k, tile_n=int(rng.choice([0, 64, 128, 256]))))
    table = g.grouped_tile_table(engine)
    want = sum(_packed_bytes(q["m"], q["n"], q["k"], q["tile_n"] or table[g.grouped_bucket(q["m"], q["n"], q["k"])],
                             np_) for q in inst)
    assert g.grouped_workspace_size(inst, engine) == want


def test_create_rejects_bad_arguments_before_device_work():
    with pytest.raises(g.GatlasError, match="status -3"):
        g.Grouped([dict(m=16, n=16, k=16)], engine="tc_split6")
    with pytest.raises(g.GatlasError, match="tile width"):
        g.Grouped([dict(m=16, n=16, k=16, tile_n=48)], engine="tc_split3")
    with pytest.raises(g.GatlasError, match="null pointer"):
        g.Grouped([dict(m=16, n=16, k=16)], engine="tc_split3")
    with pytest.raises(g.GatlasError, match="leading dimension"):
        g.Grouped([dict(m=16, n=16, k=16, lda=8)], engine="tc_split3")
    assert g.grouped_workspace_size([dict(m=-1, n=16, k=16)]) == 0


@pytest.mark.parametrize("engine", ["tc_bf16", "tc_split3"])
def test_create_asks_for_exactly_the_queried_workspace(engine, no_cuda_device):
    """A caller's workspace one byte short of the query is rejected with the
    size create needs, which is the query's; an unaligned one is rejected too
    (both before any device work)."""
    import ctypes
    import re
    rng = np.random.default_rng(7)
    inst = [dict(m=int(m), n=int(n), k=int(k)) for m, n, k in rng.integers(1, 900, (25, 3))]
    need = g.grouped_workspace_size(inst, engine)
    assert need > 0
    arr = g._grouped_instances(inst)
    for i in range(len(inst)):
        arr[i].a = arr[i].b = arr[i].c = 1 << 20   # never dereferenced: create stops at the size check
    h = ctypes.c_void_p()
    L = g.lib()
    rc = L.gatlas_grouped_create(g._engine(engine), arr, len(inst), ctypes.c_void_p(1 << 20), need - 1, ctypes.byref(h))
    assert rc == g.ERR_INVALID and not h.value
    assert int(re.search(r"workspace \d+ < (\d+) bytes", g.last_error()).group(1)) == need
    rc = L.gatlas_grouped_create(g._engine(engine), arr, len(inst), ctypes.c_void_p((1 << 20) + 256), need,
                                 ctypes.byref(h))
    assert rc == g.ERR_INVALID and "1024-byte aligned" in g.last_error()
