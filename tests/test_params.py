"""Parameter-space rules (oracle restatement) against the reference's own
printed parameter lines and journal key format (CPU)."""
import json
import os

import pytest

from oracle.params import (MATMUL_TYPES, Matmul, Matvec, Saxpy, journal_key,
                           matmul_search_space, matvec_search_space)

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
EX = json.load(open(os.path.join(GOLDEN, "reference_examples.json")))


def _kernel(t):
    v, sc, vl, _, _ = MATMUL_TYPES[t]
    return Matmul(variant=v, scalar=sc, vl=vl)


@pytest.mark.parametrize("e", EX["matmul"], ids=lambda e: e["cite"])
def test_reference_printed_points(e):
    k = _kernel(e["type"])
    k.set_params(e["params"])
    assert k.valid()                       # the reference ran it
    assert k.params() == e["params"]
    assert k.extra_param_detail() == e["extra_detail"]
    if e["gflops"] is not None:
        rate = k.number_flops() * e["trials"] / e["usec"] / 1000
        if e["trials"] == 1:
            assert rate == pytest.approx(e["gflops"], rel=5e-6)
        else:
            # mean of per-trial rates vs aggregate rate: within a few stddevs
            assert abs(rate - e["gflops"]) <= max(3 * e["stddev"] / e["trials"] ** 0.5 * 4, 1e-3 * rate)


def test_journal_key_format():
    for e in EX["journal_keys"]:
        k = _kernel(e["type"])
        k.set_params(e["params"])
        key, value = e["line"].split("\t")
        assert journal_key(k.kernel_name(), k.params()) == key
        assert int(value) == -1   # BUILD_IN_PROGRESS


def test_kernel_names():
    assert _kernel("float4").kernel_name() == "matmulbufferfloat4"
    assert _kernel("floatimg").kernel_name() == "matmulimagefloat4"
    assert _kernel("doubleimg").kernel_name() == "matmulimagedouble2"
    assert Matvec(variant="image", scalar="float", vl=4).kernel_name() == "matvecimagefloat4"
    assert Saxpy(variant="buffer", scalar="double", vl=2).kernel_name() == "saxpybufferdouble2"


def test_total_variations():
    assert _kernel("float4").total_variations() == 12
    assert _kernel("floatimg").total_variations() == 24
    assert Matvec(variant="buffer").total_variations() == 2
    assert Matvec(variant="image").total_variations() == 4
    assert Saxpy(variant="image").total_variations() == 4


def test_validity_rules():
    k = _kernel("float4")
    k.set_params([1, 0, 1024, 1024, 1024, 0, 0, 16, 16, 8, 4, 0])
    assert k.valid()
    k.set_params([1, 0, 1024, 1024, 1024, 1, 0, 16, 16, 6, 4, 0])
    assert not k.valid()               # transposed A needs block_h % VL == 0
    k.set_params([1, 0, 1024, 1024, 1024, 0, 0, 16, 16, 8, 4, 12])
    assert not k.valid()               # extra parameter out of range
    k.set_params([0, 0, 1024, 1024, 1024, 0, 0, 16, 16, 8, 4, 0])
    assert not k.valid()               # packedCalc must be > 0
    k.set_params([1, 0, 64, 64, 64, 0, 0, 16, 16, 8, 4, 0])
    assert not k.valid()               # tile 128 > M
    k.set_params([1, 0, 1024, 1024, 1024, 0, 0, 0, 16, 8, 4, 0])
    assert not k.valid()               # zero work group (a trap in the reference)


def test_matmul_search_space_shape():
    # benchMatmul getParams with everything free: largest valid square group
    # from min(maxWG, sqrt(1024)) down to 9, then group 8 (benchMatmul.cpp:258-300)
    k = _kernel("float4")
    k.M = k.N = k.K = 1024
    pts = matmul_search_space(k, 10, 10)
    groups = sorted({p[7] for p in pts})
    assert groups[0] == 8 and max(groups) <= 10
    assert all(p[10] == 4 for p in pts)          # block width == VL
    assert all(4 <= p[9] <= 10 for p in pts)      # block height VL..maxBH
    k2 = _kernel("float4")
    k2.M = k2.N = k2.K = 1024
    assert len(matmul_search_space(k2, 10, 10, group_size=16, block_height=8)) == 12


def test_matvec_search_space_shape():
    k = Matvec(variant="buffer", scalar="float", vl=4, M=16384, N=16384)
    pts = matvec_search_space(k, 64, 256)
    assert pts and all(p[7] == 4 for p in pts)
    assert min(p[5] for p in pts) == 64
