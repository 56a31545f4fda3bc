"""bench.py host plumbing on CPU: two ranks over gloo (127.0.0.1) take the
barrier, reduce their step times to the slowest rank's and report whole-job
throughput for weak scaling; under --impl reference only rank 0 works; the
clock sampler reports even where no GPU can be queried."""
import json
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import argparse

    import torch.distributed as dist

    import bench
    r, w, local = bench._dist_init(world, backend="gloo")
    bench._barrier(w)
    # rank r took 10 * (r + 1) ms for 1 TFLOP of work
    value, ms_max = bench._aggregate(1e12, 10.0 * (r + 1), w)
    ref = bench.run_reference(argparse.Namespace(steps=1, warmup=0), r, w) if r != 0 else "skipped"
    bench._barrier(w)
    with open(os.path.join(out_dir, f"rank{r}.json"), "w") as f:
        json.dump({"rank": r, "world": w, "local": local, "value": value, "ms_max": ms_max, "ref": ref}, f)
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_ranks_reduce_to_the_slowest_and_aggregate(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn",
                       join=True)
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    for r, d in enumerate(res):
        assert d["rank"] == r and d["world"] == world and d["local"] == r
        assert d["ms_max"] == pytest.approx(20.0)                     # the slowest rank's time on every rank
        assert d["value"] == pytest.approx(world * 1e12 / 20e-3 / 1e12)  # whole-job TFLOP/s
    assert res[1]["ref"] is None                                      # reference arm: rank 0 only


def test_single_process_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench._aggregate(2e12, 4.0, 1) == (pytest.approx(500.0), 4.0)
    bench._barrier(1)


def test_clock_sampler_reports_without_a_gpu():
    # with neither NVML nor nvidia-smi usable the sampler says so instead of failing
    sys.path.insert(0, ROOT)
    import bench
    s = bench.ClockSampler(0)
    s.start()
    out = s.stop()
    assert {"sm_mhz", "sm_max_mhz", "reasons"} <= set(out)
