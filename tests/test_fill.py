"""Seeded device generators: bit-identical to the oracle's counter-based
streams for every length, offset and alignment (the 16-byte path, the
unaligned path and the tail)."""
import numpy as np
import pytest

import gatlas_b200 as g
import oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("n", [1, 3, 17, 4096, 1_000_003])
@pytest.mark.parametrize("shift", [0, 1])
def test_uniform_matches_oracle(cuda, dtype, n, shift):
    import torch
    buf = torch.empty(n + shift, dtype=torch.float32 if dtype == np.float32 else torch.float64, device=cuda)
    t = buf[shift:]                                   # shift = 1: base not 16-byte aligned
    g.fill(t, "uniform", seed=9, offset=5)
    torch.cuda.synchronize()
    assert np.array_equal(t.cpu().numpy(), oracle.uniform(n, seed=9, offset=5, dtype=dtype))


@pytest.mark.parametrize("n", [7, 100_000])
def test_pow2_and_constant(cuda, n):
    import torch
    t = torch.empty(n, device=cuda)
    g.fill(t, "pow2", seed=3)
    assert np.array_equal(t.cpu().numpy(), oracle.pow2(n, seed=3))
    g.fill(t, "const", value=2.5)
    assert (t.cpu().numpy() == np.float32(2.5)).all()
