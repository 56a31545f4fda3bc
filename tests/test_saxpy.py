"""SAXPY parity: bit-exact against a per-element fmaf (oracle ORACLE_FMA)."""
import os

import numpy as np
import pytest

import gatlas_b200 as g
import oracle

pytestmark = pytest.mark.gpu
GOLDEN = np.load(os.path.join(os.path.dirname(__file__), "golden", "oracle_small.npz"))


def _run(cuda, x, y, alpha, engine, dtype, inplace=False, offset=0):
    import torch
    tdt = torch.float32 if dtype == np.float32 else torch.float64
    n = x.size
    xb = torch.zeros(n + offset, dtype=tdt, device=cuda)
    yb = torch.zeros(n + offset, dtype=tdt, device=cuda)
    xb[offset:] = torch.from_numpy(x).to(cuda)
    yb[offset:] = torch.from_numpy(y).to(cuda)
    xt, yt = xb[offset:], yb[offset:]
    out = yt if inplace else torch.empty_like(yt)
    g.saxpy(alpha, xt, yt, out=out, engine=engine)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_golden_fixture(cuda):
    for engine in ("buffer", "image"):
        z = _run(cuda, GOLDEN["sx_x"], GOLDEN["sx_y"], 0.5, engine, np.float32)
        assert np.array_equal(z, GOLDEN["sx_fma"])


@pytest.mark.parametrize("engine", ["buffer", "image"])
def test_known_answer_z_equals_two(cuda, engine):
    n = 1 << 20
    z = _run(cuda, np.ones(n, np.float32), np.ones(n, np.float32), 1.0, engine, np.float32)
    assert oracle.check_pattern(z, 2.0)


@pytest.mark.parametrize("engine", ["buffer", "image"])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("n", [0, 1, 3, 4, 5, 1023, 4096, 4097, 65537, 1_000_003, (1 << 22) + 7])
def test_bit_exact_vs_fmaf(cuda, engine, dtype, n):
    x = oracle.uniform(n, seed=100 + n % 97, dtype=dtype)
    y = oracle.uniform(n, seed=200 + n % 89, dtype=dtype)
    z = _run(cuda, x, y, 0.5 if dtype == np.float32 else 0.3, engine, dtype)
    ref = oracle.saxpy(0.5 if dtype == np.float32 else 0.3, x, y, mode=oracle.FMA, dtype=dtype)
    assert np.array_equal(z, ref)


@pytest.mark.parametrize("engine", ["buffer", "image"])
@pytest.mark.parametrize("offset", [1, 2, 3])
def test_misaligned_and_in_place(cuda, engine, offset):
    n = 100_003
    x = oracle.uniform(n, seed=7)
    y = oracle.uniform(n, seed=8)
    z = _run(cuda, x, y, -1.75, engine, np.float32, inplace=True, offset=offset)
    assert np.array_equal(z, oracle.saxpy(-1.75, x, y, mode=oracle.FMA))


@pytest.mark.parametrize("engine", ["buffer", "image"])
def test_full_size_in_place(cuda, engine):
    # the memory-bound workload's full size: n = 2^28 (1 GiB per operand),
    # in place, checked element by element against fmaf
    import torch
    n = 1 << 28
    x = torch.empty(n, dtype=torch.float32, device=cuda)
    y = torch.empty(n, dtype=torch.float32, device=cuda)
    g.fill(x, "uniform", seed=1)
    g.fill(y, "uniform", seed=2)
    g.saxpy(0.5, x, y, out=y, engine=engine)
    got = y.cpu().numpy()
    ref = oracle.saxpy(0.5, oracle.uniform(n, 1), oracle.uniform(n, 2), mode=oracle.FMA)
    assert np.array_equal(got, ref)
    assert g.device_faults() == 0
