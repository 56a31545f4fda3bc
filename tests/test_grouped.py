"""Grouped GEMM on the GPU: one persistent tcgen05 launch over uneven
instances.  Every instance's result is bit-identical to the single-instance
engine's (same BF16 pieces, same MMA order, same promotion), whatever the
tile width, the other instances in the group or the launch path (direct or
CUDA graph), and within the engine's FP64 error budget."""
import numpy as np
import pytest

import gatlas_b200 as g
import oracle

pytestmark = pytest.mark.gpu
BUDGET = {"tc_bf16": 2.0 ** -7, "tc_split3": 8e-6}


def _make(cuda, shapes, seed=1):
    """shapes: (m, n, k, ta, tb, gemm, alpha, beta, tile_n).  Returns instances with
    host copies of the inputs."""
    import torch
    inst = []
    for i, (m, n, k, ta, tb, gemm, alpha, beta, tn) in enumerate(shapes):
        A = oracle.uniform(m * k, seed=seed + 3 * i)
        B = oracle.uniform(k * n, seed=seed + 3 * i + 1)
        C0 = oracle.uniform(m * n, seed=seed + 3 * i + 2)
        inst.append(dict(A=torch.from_numpy(A).to(cuda), B=torch.from_numpy(B).to(cuda),
                         C=torch.from_numpy(C0.copy()).to(cuda), m=m, n=n, k=k, trans_a=ta, trans_b=tb,
                         gemm=gemm, alpha=alpha, beta=beta, tile_n=tn, hA=A, hB=B, hC0=C0))
    return inst


def _reset(inst):
    import torch
    for q in inst:
        q["C"].copy_(torch.from_numpy(q["hC0"]))


def _results(inst):
    import torch
    torch.cuda.synchronize()
    assert g.device_faults() == 0
    return [q["C"].cpu().numpy().copy() for q in inst]


SHAPES = [
    (128, 256, 64, 0, 0, 0, 1.0, 0.0, 0), (200, 300, 100, 0, 1, 1, 0.5, 1.0, 0), (33, 17, 5, 1, 0, 0, 1.0, 0.0, 64),
    (257, 129, 520, 1, 1, 1, 2.0, 0.0, 128), (16, 4000, 48, 0, 0, 1, 1.5, 1.0, 256), (1000, 16, 700, 1, 0, 0, 1.0, 0.0, 0),
    (64, 64, 1, 0, 1, 0, 1.0, 0.0, 64), (300, 500, 0, 0, 0, 1, 1.0, 0.5, 0), (0, 50, 50, 0, 0, 0, 1.0, 0.0, 0),
    (130, 70, 90, 1, 1, 1, 0.75, 1.0, 128), (512, 512, 256, 0, 0, 0, 1.0, 0.0, 256), (96, 1024, 33, 1, 0, 1, 1.0, 1.0, 0),
]


@pytest.mark.parametrize("engine", ["tc_bf16", "tc_split3"])
def test_grouped_equals_single_instance_engine(cuda, engine):
    inst = _make(cuda, SHAPES)
    plan = g.Grouped(inst, engine=engine)
    plan.prepare().run()
    got = _results(inst)
    _reset(inst)
    plan.run_each()
    want = _results(inst)
    for q, x, y in zip(inst, got, want):
        assert np.array_equal(x, y), (q["m"], q["n"], q["k"])
        if q["m"] and q["n"]:
            ref = oracle.matmul(q["hA"], q["hB"], q["m"], q["n"], q["k"], q["trans_a"], q["trans_b"], mode=oracle.F64,
                                gemm=q["gemm"], Cin=q["hC0"], alpha=q["alpha"], beta=q["beta"])
            assert oracle.normwise_error(x, ref) <= BUDGET[engine]
    info = plan.info()
    assert info["ctas"] <= 148 and info["tiles"] > 0
    plan.close()


# every C takes 8-byte vector accesses (even n): the launch runs the
# vector-only epilogue; ragged tiles in both dimensions, beta in {0, 1}
EVEN_SHAPES = [
    (128, 256, 64, 0, 0, 0, 1.0, 0.0, 0), (200, 300, 100, 0, 1, 1, 0.5, 1.0, 0), (33, 18, 5, 1, 0, 1, 1.0, 1.0, 64),
    (257, 130, 520, 1, 1, 1, 2.0, 0.0, 128), (16, 4000, 48, 0, 0, 1, 1.5, 1.0, 256), (1000, 16, 700, 1, 0, 0, 1.0, 0.0, 0),
    (130, 70, 90, 1, 1, 1, 0.75, 1.0, 128), (96, 1022, 33, 1, 0, 1, 1.0, 1.0, 0), (300, 500, 0, 0, 0, 1, 1.0, 0.5, 0),
]


@pytest.mark.parametrize("engine", ["tc_bf16", "tc_split3"])
@pytest.mark.parametrize("pair", [0, 1])
def test_vector_epilogue_equals_single_instance_engine(cuda, engine, pair, pair_option):
    g.set_option("grouped_pair", pair)
    inst = _make(cuda, EVEN_SHAPES, seed=11)
    plan = g.Grouped(inst, engine=engine)
    plan.prepare().run()
    got = _results(inst)
    _reset(inst)
    plan.run_each()
    want = _results(inst)
    for q, x, y in zip(inst, got, want):
        assert np.array_equal(x, y), (q["m"], q["n"], q["k"])
        if q["m"] and q["n"]:
            ref = oracle.matmul(q["hA"], q["hB"], q["m"], q["n"], q["k"], q["trans_a"], q["trans_b"], mode=oracle.F64,
                                gemm=q["gemm"], Cin=q["hC0"], alpha=q["alpha"], beta=q["beta"])
            assert oracle.normwise_error(x, ref) <= BUDGET[engine]
    plan.close()


@pytest.fixture
def pair_option():
    old = g.get_option("grouped_pair")
    yield
    g.set_option("grouped_pair", old)


@pytest.mark.parametrize("engine", ["tc_bf16", "tc_split3"])
def test_cta_pairs_equal_single_ctas(cuda, engine, pair_option):
    # 256-row tiles on CTA pairs against 128-row tiles on single CTAs: odd and
    # even counts of row blocks, every tile width, ragged edges
    rng = np.random.default_rng(21)
    shapes = SHAPES + [(int(rng.integers(1, 900)), int(rng.integers(1, 700)), int(rng.integers(1, 400)),
                        int(rng.integers(0, 2)), int(rng.integers(0, 2)), int(rng.integers(0, 2)), 1.25,
                        float(rng.integers(0, 2)), int(rng.choice([0, 64, 128, 256]))) for _ in range(24)]
    inst = _make(cuda, shapes, seed=21)
    g.set_option("grouped_pair", 0)
    single = g.Grouped(inst, engine=engine)
    single.prepare().run()
    want = _results(inst)
    g.set_option("grouped_pair", 1)
    pair = g.Grouped(inst, engine=engine)
    assert pair.info()["ctas"] % 2 == 0 and pair.info()["tiles"] < single.info()["tiles"]
    for launch in (lambda: pair.prepare().run(), lambda: pair.launch_graph(with_prepare=True)):
        _reset(inst)
        launch()
        for q, x, y in zip(inst, _results(inst), want):
            assert np.array_equal(x, y), (q["m"], q["n"], q["k"], q["tile_n"])
    single.close()
    pair.close()


@pytest.mark.parametrize("tile_n", [64, 128, 256])
def test_result_independent_of_tile_width(cuda, tile_n):
    shapes = [(200, 300, 100, 0, 1, 1, 0.5, 1.0, tile_n), (77, 45, 260, 1, 0, 0, 1.0, 0.0, tile_n)]
    inst = _make(cuda, shapes, seed=5)
    g.Grouped(inst, engine="tc_split3").prepare().run()
    got = _results(inst)
    _reset(inst)
    for q in inst:
        q["tile_n"] = 256
    g.Grouped(inst, engine="tc_split3").prepare().run()
    assert all(np.array_equal(x, y) for x, y in zip(got, _results(inst)))


def test_same_result_alone_and_in_the_mix(cuda):
    rng = np.random.default_rng(3)
    shapes = [(int(rng.integers(16, 600)), int(rng.integers(16, 600)), int(rng.integers(16, 600)),
               int(rng.integers(0, 2)), int(rng.integers(0, 2)), 1, 1.0, float(rng.integers(0, 2)), 0)
              for _ in range(60)]
    inst = _make(cuda, shapes, seed=9)
    g.Grouped(inst, engine="tc_split3").prepare().run()
    mixed = _results(inst)
    for i in (0, 17, 59):
        _reset(inst)
        g.Grouped([inst[i]], engine="tc_split3").prepare().run()
        assert np.array_equal(_results([inst[i]])[0], mixed[i])


def test_graph_launch_matches_direct_and_replays(cuda):
    inst = _make(cuda, SHAPES[:6], seed=11)
    plan = g.Grouped(inst, engine="tc_split3")
    plan.prepare().run()
    direct = _results(inst)
    for _ in range(3):
        _reset(inst)
        plan.launch_graph(with_prepare=True)
        assert all(np.array_equal(x, y) for x, y in zip(direct, _results(inst)))
    _reset(inst)
    plan.launch_graph(with_prepare=False)          # packed operands are still resident
    assert all(np.array_equal(x, y) for x, y in zip(direct, _results(inst)))


def test_caller_workspace(cuda):
    import torch
    inst = _make(cuda, SHAPES[:4], seed=13)
    need = g.grouped_workspace_size(inst, "tc_split3")
    ws = torch.empty(need + 1024, dtype=torch.uint8, device=cuda)
    ws = ws[(-ws.data_ptr()) % 1024:][:need]
    g.Grouped(inst, engine="tc_split3", workspace=ws).prepare().run()
    got = _results(inst)
    _reset(inst)
    g.Grouped(inst, engine="tc_split3").prepare().run()
    assert all(np.array_equal(x, y) for x, y in zip(got, _results(inst)))
    with pytest.raises(g.GatlasError):
        g.Grouped(inst, engine="tc_split3", workspace=ws[:1024])


def test_autotune_journals_and_replays(cuda, tmp_path):
    from oracle.params import BUILD_IN_PROGRESS, BUILD_OK, RUN_IN_PROGRESS, RUN_OK
    j = tmp_path / "grouped.journal"
    old = g.grouped_tile_table("tc_bf16")
    try:
        table = g.grouped_autotune("tc_bf16", journal=str(j), trials=1, seed=3)
        assert all(t in (64, 128, 256) for t in table)
        lines = [ln.split("\t") for ln in j.read_text().splitlines()]
        assert len(lines) % 5 == 0 and 4 * 2 * 5 <= len(lines) <= 4 * 3 * 5   # a repeated table is replayed
        assert [int(v) for _, v in lines[:4]] == [BUILD_IN_PROGRESS, BUILD_OK, RUN_IN_PROGRESS, RUN_OK]
        t0 = old
        assert lines[0][0] == "groupedtcbf16_0_64_192_3_64_%d_%d_%d_" % tuple(t0[1:])
        # resumed: every timing replayed from the journal, same decision
        n = len(lines)
        g.grouped_tile_table("tc_bf16", old)
        assert g.grouped_autotune("tc_bf16", journal=str(j), trials=1, seed=3) == table
        assert len(j.read_text().splitlines()) == n
    finally:
        g.grouped_tile_table("tc_bf16", old)
