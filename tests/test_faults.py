"""The bounded-wait mechanism every TMA / tcgen05 kernel relies on, exercised
without faulting the GPU: a wait on an mbarrier that nothing completes runs
out after its limit, sets the fault word and returns, and the device keeps
working; a completed wait leaves the word clear."""
import numpy as np
import pytest

import gatlas_b200 as g
import oracle


@pytest.mark.gpu
def test_wait_that_nothing_completes_reports_and_returns(cuda):
    import torch
    g.device_faults(clear=True)
    assert g.selftest_bounded_wait(limit_ns=1_000_000, arrive=True) is True
    assert g.device_faults(clear=True) == 0
    assert g.selftest_bounded_wait(limit_ns=1_000_000, arrive=False) is False
    assert g.device_faults(clear=True) & g.FAULT_SELFTEST_WAIT
    # the context is intact: a kernel afterwards still runs and checks out
    x, y = oracle.uniform(1000, seed=1), oracle.uniform(1000, seed=2)
    z = g.saxpy(0.5, torch.from_numpy(x).to(cuda), torch.from_numpy(y).to(cuda)).cpu().numpy()
    assert np.array_equal(z, oracle.saxpy(0.5, x, y, mode=oracle.FMA))
    assert g.device_faults(clear=True) == 0


def test_limits_are_checked_before_any_device_work():
    with pytest.raises(g.GatlasError, match="limit"):
        g.selftest_bounded_wait(limit_ns=0)
    with pytest.raises(g.GatlasError, match="limit"):
        g.selftest_bounded_wait(limit_ns=5_000_000_000)
