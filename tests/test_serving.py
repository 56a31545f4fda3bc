"""Serving loop on the GPU: continuous batching of mixed GEMM / GEMV / SAXPY
requests under a device-memory budget.  Every request's result is the same
in the mix (continuous mode, batched with others) and alone (serial mode,
one engine call), bit for bit, and matches the oracle on the inputs its seed
generates; admission never exceeds the budget."""
import numpy as np
import pytest

import gatlas_b200 as g
import oracle

pytestmark = pytest.mark.gpu
SPLIT3_BUDGET = 8e-6


def _trace(n, seed=1, burst=True, rate=5000.0, gemm_hi=600, gemv_hi=3000):
    rng = np.random.default_rng(seed)
    req = np.zeros(n, dtype=g.request_dtype())
    kinds = rng.choice([g.REQ_GEMM, g.REQ_GEMV, g.REQ_SAXPY], n, p=[0.6, 0.3, 0.1])
    lu = lambda lo, hi: int(round(np.exp(rng.uniform(np.log(lo), np.log(hi)))))
    t = 0.0
    for i in range(n):
        r = req[i]
        r["kind"] = kinds[i]
        r["seed"] = 1000 + i
        r["retain"] = 1
        if kinds[i] == g.REQ_GEMM:
            r["m"], r["n"], r["k"] = lu(16, gemm_hi), lu(16, gemm_hi), lu(16, gemm_hi)
            r["trans_a"], r["trans_b"] = rng.integers(0, 2), rng.integers(0, 2)
            r["alpha"], r["beta"] = rng.uniform(0.5, 2.0), float(rng.integers(0, 2))
        elif kinds[i] == g.REQ_GEMV:
            r["m"], r["n"] = lu(64, gemv_hi), lu(64, gemv_hi)
            r["trans_a"] = rng.integers(0, 2)
            r["alpha"], r["beta"] = 1.0, float(rng.integers(0, 2))
        else:
            r["n"] = lu(1 << 10, 1 << 18)
            r["alpha"] = 0.5
        if not burst:
            t += rng.exponential(1.0 / rate)
        r["arrival_ns"] = int(t * 1e9)
    return req


def _results(srv, req, out):
    vals = []
    for i in range(len(req)):
        assert out[i]["status"] == 0, (i, g.last_error())
        vals.append(srv.read(out[i]))
        srv.release(out[i])
    return vals


@pytest.mark.parametrize("burst", [True, False])
def test_same_result_in_the_mix_and_alone(cuda, burst):
    req = _trace(40, seed=3, burst=burst)
    srv = g.Server(2 << 30)
    mixed_out = srv.run(req, "continuous")
    mixed = _results(srv, req, mixed_out)
    alone = _results(srv, req, srv.run(req, "serial"))
    for i, (a, b) in enumerate(zip(mixed, alone)):
        assert np.array_equal(a, b), (i, req[i])
    gemm_batches = {int(b) for b, k in zip(mixed_out["batch"], req["kind"]) if k == g.REQ_GEMM}
    assert -1 not in gemm_batches
    st = srv.stats()
    assert st["used_bytes"] == 0 and st["peak_bytes"] <= st["budget_bytes"]
    if burst:
        assert st["gemm_batches"] < st["batched_gemms"]   # the burst was batched
    srv.close()


def test_results_match_the_oracle(cuda):
    req = _trace(24, seed=5)
    srv = g.Server(2 << 30)
    out = srv.run(req, "continuous")
    res = _results(srv, req, out)
    for r, y in zip(req, res):
        s = int(r["seed"]) * 4
        m, n, k = int(r["m"]), int(r["n"]), int(r["k"])
        if r["kind"] == g.REQ_GEMM:
            A, B = oracle.uniform(m * k, seed=s), oracle.uniform(k * n, seed=s + 1)
            C0 = oracle.uniform(m * n, seed=s + 2) if r["beta"] else np.zeros(m * n, np.float32)
            ref = oracle.matmul(A, B, m, n, k, int(r["trans_a"]), int(r["trans_b"]), mode=oracle.F64, gemm=1,
                                Cin=C0, alpha=float(r["alpha"]), beta=float(r["beta"]))
            assert oracle.normwise_error(y, ref) <= SPLIT3_BUDGET
        elif r["kind"] == g.REQ_GEMV:
            A, x = oracle.uniform(m * n, seed=s), oracle.uniform(n, seed=s + 1)
            y0 = oracle.uniform(m, seed=s + 2) if r["beta"] else np.zeros(m, np.float32)
            ref = oracle.matvec(A, x, m, n, int(r["trans_a"]), mode=oracle.F64, gemv=1, cin=y0,
                                alpha=float(r["alpha"]), beta=float(r["beta"]))
            assert oracle.normwise_error(y, ref) <= 4 * n * 2.0 ** -24
        else:
            x, y0 = oracle.uniform(n, seed=s), oracle.uniform(n, seed=s + 2)
            assert np.array_equal(y, oracle.saxpy(float(r["alpha"]), x, y0, mode=oracle.FMA))


def test_admission_waits_for_memory(cuda):
    # ten 512x512x512 GEMMs (about 5 MiB each with packed pieces) under a
    # 12 MiB budget: at most two are resident at once
    req = np.zeros(10, dtype=g.request_dtype())
    req["kind"] = g.REQ_GEMM
    req["m"] = req["n"] = req["k"] = 512
    req["alpha"] = 1.0
    req["seed"] = np.arange(10)
    srv = g.Server(12 << 20)
    out = srv.run(req, "continuous")
    assert (out["status"] == 0).all()
    st = srv.stats()
    assert st["peak_bytes"] <= 12 << 20 and st["used_bytes"] == 0
    order = np.argsort(out["admit_ns"], kind="stable")
    assert (order == np.arange(10)).all()                       # FIFO: nobody overtakes
    assert out["admit_ns"][9] >= out["done_ns"][0]              # the last waited for memory


def test_oversized_request_is_rejected_and_the_rest_served(cuda):
    req = _trace(6, seed=7)
    req["retain"] = 0
    req[2]["kind"], req[2]["n"] = g.REQ_SAXPY, 1 << 24       # 128 MiB > budget
    srv = g.Server(64 << 20)
    out = srv.run(req, "continuous")
    assert out[2]["status"] == -5                            # GATLAS_ERR_NOMEM
    assert all(out[i]["status"] == 0 for i in range(6) if i != 2)
    assert srv.stats()["used_bytes"] == 0


def test_latency_accounting_on_a_poisson_trace(cuda):
    req = _trace(60, seed=9, burst=False, rate=2000.0)
    req["retain"] = 0
    srv = g.Server(2 << 30)
    for mode in ("continuous", "serial"):
        out = srv.run(req, mode)
        assert (out["status"] == 0).all()
        assert (out["admit_ns"] >= req["arrival_ns"]).all()
        # the device clock starts no later than the host clock: completions never
        # precede their admission on the host's timeline
        assert (out["done_ns"] >= out["admit_ns"]).all()
    with pytest.raises(g.GatlasError):
        srv.release({"result": 12345})
