#!/usr/bin/env python
"""Benchmark of the GATLAS hot path on B200.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step is one pass of the hot path over one batch of synthetic input:
  * headline  : SGEMM at FP32 accuracy, C = A·B, M = N = K = 8192, FP32
                operands uniform[-1,1) (the precision-sweep workload), on the
                FP32-accurate engine (split-BF16 tensor cores when built,
                otherwise the SIMT kernel);
  * secondary : the memory-bound pair at full size, SGEMV y = A·x and
                y = A^T·x with A 16384^2 and SAXPY y = 0.5·x + y with n = 2^28,
                reported in GB/s against measured HBM bandwidth.
Every operand is larger than the 126 MB L2, so no flush is needed between
timed iterations.  Timing uses CUDA events on the launching stream, max over
ranks; N > 1 runs independent replicas (weak scaling, no collective on the
data path).  Rank 0 prints one JSON line.

--impl reference times the reference's own kernels on the host cores: its
generated OpenCL C buffer matmul, emitted by the reference's generators and
compiled for the host CPU (oracle/_ref), on a bounded sample of the same
workload per step (bands of work groups of the 8192^3 product).  Where
oracle/_ref is absent the oracle's port of the same algorithm stands in.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

M_GEMM = 8192
N_GEMV = 16384
N_SAXPY = 1 << 28
METRIC = "SGEMM TFLOP/s at FP32 accuracy (3xBF16 TC vs SIMT FP32); GEMV GB/s; p99 lat"


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return {"hbm_gbs": float(d["hbm_gbs"]), "bf16_tflops": float(d["bf16_tflops"]),
                "bf16_tflops_sustained": float(d.get("bf16_tflops_sustained", d["bf16_tflops"])),
                "source": "measured"}
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0,
                "source": "fallback"}


# DRAM bytes (read + write) per launch of the split3 contraction at 8192^3
# (persistent kernel on CTA pairs, A's loads evict-last), from an ncu capture
# of the full-size launch (profiles/tc_gemm_persistent_split3_pair_8192.md)
TC_TRAFFIC_BYTES = 2.542e9 + 0.263e9
TC_KERNEL = "tc_gemm_persistent_kernel<split3, CTA pair>"

# nominal FP32 SIMT peak: 148 SMs x 128 FP32 lanes x 2 flop x 1.965 GHz
FP32_SIMT_NOMINAL_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12


class ClockSampler:
    """Samples the SM clock, power and clock-event (throttle) reasons of one GPU
    every 10 ms through NVML while the timed region runs; falls back to
    `nvidia-smi -lms 200` where NVML is unavailable."""

    # NVML clock-event reason bits (nvml.h)
    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
               0x80: "hw_power_brake_slowdown"}
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.samples: list[tuple[float, float, int]] = []  # (sm MHz, W, reason bits)
        self.smax = None
        self._stop = threading.Event()
        self._t = None
        self.proc = None
        self.lines: list[str] = []
        self.nvml = None

    def _handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.dev).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID("GPU-" + uuid)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.dev)

    def start(self):
        try:
            nv, h = self._handle()
            self.nvml = (nv, h)
            self.smax = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons

            def poll():
                while not self._stop.is_set():
                    try:
                        self.samples.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                                             nv.nvmlDeviceGetPowerUsage(h) / 1000.0, int(reasons(h))))
                    except Exception:
                        pass
                    self._stop.wait(0.01)
            self._t = threading.Thread(target=poll, daemon=True)
            self._t.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self._t = threading.Thread(target=lambda: self.lines.extend(ln.strip() for ln in self.proc.stdout),
                                   daemon=True)
        self._t.start()

    def stop(self) -> dict:
        if self.nvml is not None:
            self._stop.set()
            if self._t:
                self._t.join(timeout=2)
            sm = [x[0] for x in self.samples]
            bits = 0
            for x in self.samples:
                bits |= x[2]
            reasons = sorted(nm for b, nm in self.REASONS.items() if bits & b)
            return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.smax,
                    "reasons": reasons, "samples": len(sm),
                    "power_w_max": max((x[1] for x in self.samples), default=None), "source": "nvml, 10 ms"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self._t:
            self._t.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi, 200 ms"}


# ---------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------

def _dist_init(n_gpus: int, backend: str = "nccl"):
    """One process per GPU: rank, world size and local rank from the launcher's
    environment; a process group (short timeout) when world > 1."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return rank, world, local


def _barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def _max_over_ranks(x: float, world: int) -> float:
    """Max of a per-rank time over all ranks (GPU tensor under NCCL, CPU under gloo)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _aggregate(flops_per_rank: float, ms_per_rank: float, world: int) -> tuple[float, float]:
    """Weak scaling: (whole-job TFLOP/s, ms_max).  Every rank does the same work;
    the job's time is the slowest rank's."""
    ms_max = _max_over_ranks(ms_per_rank, world)
    return world * flops_per_rank / (ms_max * 1e-3) / 1e12, ms_max


# ---------------------------------------------------------------------------
# our implementation
# ---------------------------------------------------------------------------

HEADLINE_ENGINE = "tc_split3"     # FP32 operands as BF16 hi/lo, 3 products, FP32 accumulation
PRODUCTS = {"tc_bf16": 1, "tc_split3": 3, "tc_split6": 6}
SWEEP_ENGINES = ("buffer", "tc_bf16", "tc_split3", "tc_split6", "tc_fp8")


def _timed(fn, steps, warmup, world, stream, sampler=None):
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    _barrier(world)
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    if sampler is not None:
        sampler.start()  # samples exactly the timed launches
    start.record(stream)
    for _ in range(steps):
        fn()
    stop.record(stream)
    torch.cuda.synchronize()
    if sampler is not None:
        sampler.clocks = sampler.stop()
    _barrier(world)
    return start.elapsed_time(stop) / steps  # ms per step


SGEMM_TUNE_N = 1024
SGEMM_TUNE_GRID = [(gh, gw, bh, bw, vl) for gh in (8, 16) for gw in (8, 16) for bh in (4, 8) for bw in (4, 8)
                   for vl in (1, 2, 4)]


def sgemm_autotune_leg(world, stream):
    """Plain SGEMM 1024^3 (alpha 1, beta 0, row-major, no transposes) on the
    SIMT engine, autotuned over work group {8,16}^2 x inner blocking {4,8}^2 x
    vector width {1,2,4}; the winner is checked against the FP64 product."""
    import torch

    import gatlas_b200 as g
    dev = torch.cuda.current_device()
    n = SGEMM_TUNE_N
    A = torch.empty(n * n, device=dev)
    B = torch.empty(n * n, device=dev)
    C = torch.empty(n * n, device=dev)
    g.fill(A, "uniform", seed=1)
    g.fill(B, "uniform", seed=2)
    times = {}
    for pt in SGEMM_TUNE_GRID:
        tile = pt + (0,)
        times[pt] = _timed(lambda: g.matmul(A, B, n, n, n, C=C, tile=tile), 10, 3, world, stream)
    best = min(times, key=times.get)
    g.matmul(A, B, n, n, n, C=C, tile=best + (0,))
    fro, ref, mx, _ = g.residual(A, B, C, n, n, n)
    flops = 2.0 * n ** 3
    ranked = sorted(times.items(), key=lambda kv: kv[1])
    return {"m": n, "n": n, "k": n, "points": len(times), "best_tile": dict(zip(("gh", "gw", "bh", "bw", "vl"), best)),
            "best_ms": times[best], "best_tflops": flops / (times[best] * 1e-3) / 1e12,
            "reference_flops": float(n * n * (2 * n - 1)),
            "worst_tflops": flops / (ranked[-1][1] * 1e-3) / 1e12,
            "top5": [{"tile": list(k), "tflops": flops / (v * 1e-3) / 1e12} for k, v in ranked[:5]],
            "error_vs_fp64": {"normwise": fro / ref, "max_abs": mx}}


GROUPED_INSTANCES = 1024


def grouped_workload(dev, count=GROUPED_INSTANCES, seed=4, lo=16, hi=4096):
    """The batched uneven workload: m, n, k log-uniform in [lo, hi] rounded to
    multiples of 16, random layouts, alpha uniform [0.5, 2], beta in {0, 1}.
    Operands live in three device buffers (instance offsets 64-byte aligned),
    filled with seeded uniform[-1,1) values."""
    import numpy as np
    import torch

    import gatlas_b200 as g
    rng = np.random.default_rng(seed)

    def lu(n):
        v = np.exp(rng.uniform(np.log(lo), np.log(hi), n))
        return np.clip(np.round(v / 16) * 16, lo, hi).astype(np.int64)
    m, n, k = lu(count), lu(count), lu(count)
    ta, tb = rng.integers(0, 2, count), rng.integers(0, 2, count)
    alpha, beta = rng.uniform(0.5, 2.0, count), rng.integers(0, 2, count).astype(float)
    r16 = lambda x: (int(x) + 15) // 16 * 16
    sa, sb, sc = (sum(r16(a * b) for a, b in zip(x, y)) for x, y in ((m, k), (k, n), (m, n)))
    A = torch.empty(sa, device=dev)
    B = torch.empty(sb, device=dev)
    C = torch.empty(sc, device=dev)
    g.fill(A, "uniform", seed=seed + 1)
    g.fill(B, "uniform", seed=seed + 2)
    g.fill(C, "uniform", seed=seed + 3)
    inst, oa, ob, oc = [], 0, 0, 0
    for i in range(count):
        mi, ni, ki = int(m[i]), int(n[i]), int(k[i])
        inst.append(dict(A=A[oa:oa + mi * ki], B=B[ob:ob + ki * ni], C=C[oc:oc + mi * ni], m=mi, n=ni, k=ki,
                         trans_a=int(ta[i]), trans_b=int(tb[i]), gemm=1, alpha=float(alpha[i]),
                         beta=float(beta[i])))
        oa, ob, oc = oa + r16(mi * ki), ob + r16(ki * ni), oc + r16(mi * ni)
    return inst, (A, B, C)


def grouped_leg(args, world, stream):
    """Batched uneven GEMM: one persistent grouped launch per dtype in a CUDA
    graph vs one engine call per instance."""
    import tempfile

    import numpy as np
    import torch

    import gatlas_b200 as g
    dev = torch.cuda.current_device()
    out = {"instances": GROUPED_INSTANCES, "shapes": "m, n, k log-uniform [16, 4096], multiples of 16",
           "layouts": "trans_a, trans_b random", "alpha": "uniform [0.5, 2]", "beta": "{0, 1}"}
    inst, bufs = grouped_workload(dev)
    flops = sum(2.0 * q["m"] * q["n"] * q["k"] for q in inst)
    out["gflop"] = flops / 1e9
    for eng in ("tc_split3", "tc_bf16"):
        t0 = time.time()
        with tempfile.TemporaryDirectory() as d:
            table = g.grouped_autotune(eng, journal=os.path.join(d, "grouped.journal"), trials=2, seed=1)
        row = {"tile_table": table, "autotune_s": time.time() - t0}
        plan = g.Grouped(inst, engine=eng)
        row.update(plan.info())
        C0 = bufs[2].clone()
        full = _timed(lambda: plan.launch_graph(with_prepare=True), max(3, min(args.steps, 10)), 2, world, stream)
        run = _timed(lambda: plan.launch_graph(with_prepare=False), max(3, min(args.steps, 10)), 2, world, stream)
        each = _timed(lambda: plan.run_each(), 2, 1, world, stream)
        # the per-instance path gives the same results (same pieces, same MMA order)
        sample = (0, 511, GROUPED_INSTANCES - 1)
        bufs[2].copy_(C0)
        plan.launch_graph(with_prepare=True)
        torch.cuda.synchronize()
        got = [inst[i]["C"].clone() for i in sample]
        bufs[2].copy_(C0)
        plan.run_each()
        torch.cuda.synchronize()
        same = all(torch.equal(inst[i]["C"], x) for i, x in zip(sample, got))
        del C0
        row.update({"graph_prepare_run_ms": full, "graph_run_ms": run, "per_instance_ms": each,
                    "tflops_graph_prepare_run": flops / (full * 1e-3) / 1e12,
                    "tflops_graph_run": flops / (run * 1e-3) / 1e12,
                    "tflops_per_instance": flops / (each * 1e-3) / 1e12,
                    "speedup_vs_per_instance": each / full, "bit_identical_sample": bool(same)})
        plan.close()
        out[eng] = row
    del inst, bufs
    return out


SERVE_RATES = (1000.0, 10000.0, 100000.0)
SERVE_STREAM = 100000         # requests in the full stream
SERVE_SECONDS = 4.0           # arrivals replayed per rate: min(stream, rate x seconds)
SERVE_BUDGET = 128 << 30      # device-memory admission budget


def serving_trace(count, rate, seed):
    """Poisson arrivals at `rate`/s; 60% GEMM (m, n, k log-uniform [64, 8192]),
    30% GEMV (rows, cols log-uniform [1024, 32768]), 10% SAXPY (n log-uniform
    [2^16, 2^26]); operands uniform[-1,1) from the per-request seed."""
    import numpy as np

    import gatlas_b200 as g
    rng = np.random.default_rng(seed)
    req = np.zeros(count, dtype=g.request_dtype())
    kinds = rng.choice([g.REQ_GEMM, g.REQ_GEMV, g.REQ_SAXPY], count, p=[0.6, 0.3, 0.1])
    lu = lambda lo, hi: np.round(np.exp(rng.uniform(np.log(lo), np.log(hi), count))).astype(np.int64)
    gm, gn, gk = lu(64, 8192), lu(64, 8192), lu(64, 8192)
    vm, vn = lu(1024, 32768), lu(1024, 32768)
    sn = lu(1 << 16, 1 << 26)
    ta, tb = rng.integers(0, 2, count), rng.integers(0, 2, count)
    is_mm, is_mv, is_ax = kinds == g.REQ_GEMM, kinds == g.REQ_GEMV, kinds == g.REQ_SAXPY
    req["kind"] = kinds
    req["seed"] = seed * 1000003 + np.arange(count)
    req["arrival_ns"] = (np.cumsum(rng.exponential(1.0 / rate, count)) * 1e9).astype(np.int64)
    req["m"] = np.where(is_mm, gm, np.where(is_mv, vm, 0))
    req["n"] = np.where(is_mm, gn, np.where(is_mv, vn, sn))
    req["k"] = np.where(is_mm, gk, 0)
    req["trans_a"] = np.where(is_ax, 0, ta)
    req["trans_b"] = np.where(is_mm, tb, 0)
    req["alpha"] = np.where(is_ax, 0.5, 1.0)
    return req


def _serve_stats(req, out):
    import numpy as np
    ok = out["status"] == 0
    lat = (out["done_ns"] - req["arrival_ns"])[ok] / 1e6
    span = (out["done_ns"][ok].max() - req["arrival_ns"].min()) / 1e9
    m, n, k = (req[f][ok].astype(np.float64) for f in ("m", "n", "k"))
    kind = req["kind"][ok]
    flops = float(np.where(kind == 0, 2 * m * n * k, np.where(kind == 1, 2 * m * n, 2 * n)).sum())
    return {"completed": int(ok.sum()), "failed": int((~ok).sum()), "makespan_s": span,
            "throughput_rps": float(ok.sum()) / span, "tflops": flops / span / 1e12,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean())}


def serving_leg(args):
    """Continuous batching vs a serial launch-per-request loop, per arrival rate."""
    import gatlas_b200 as g
    srv = g.Server(SERVE_BUDGET, engine="tc_split3")
    out = {"budget_bytes": SERVE_BUDGET, "gemm_engine": "tc_split3",
           "mix": "60% GEMM [64,8192]^3, 30% GEMV [1024,32768]^2, 10% SAXPY [2^16,2^26], log-uniform",
           "sample": f"the first min({SERVE_STREAM}, rate x {SERVE_SECONDS:g} s) Poisson arrivals per rate"}
    warm = serving_trace(200, 20000.0, seed=5)
    for mode in ("continuous", "serial"):
        srv.run(warm, mode)
    for i, rate in enumerate(SERVE_RATES):
        count = int(min(SERVE_STREAM, rate * SERVE_SECONDS))
        req = serving_trace(count, rate, seed=7 + i)
        row = {"requests": count}
        for mode in ("continuous", "serial"):
            st0 = srv.stats()
            res = srv.run(req, mode)
            row[mode] = _serve_stats(req, res)
            if mode == "continuous":
                st = srv.stats()
                row[mode]["gemm_batches"] = st["gemm_batches"] - st0["gemm_batches"]
                row[mode]["peak_bytes"] = st["peak_bytes"]
                row[mode]["host_busy_s"] = (st["host_busy_ns"] - st0["host_busy_ns"]) / 1e9
                row[mode]["host_phase_s"] = dict(zip(("harvest", "admit", "single_launch", "batch_tables",
                                                      "batch_launch"),
                                                     ((a - b) / 1e9 for a, b in zip(st["phase_ns"], st0["phase_ns"]))))
                # admission's operand-generation launches: time blocked in them
                # (a full device launch queue) against their count
                gl = st["generate_launches"] - st0["generate_launches"]
                gs = (st["generate_ns"] - st0["generate_ns"]) / 1e9
                row[mode]["admit_generate_s"] = gs
                row[mode]["admit_generate_us_per_launch"] = gs * 1e6 / gl if gl else None
        row["throughput_ratio"] = row["continuous"]["throughput_rps"] / row["serial"]["throughput_rps"]
        row["p50_ratio"] = row["serial"]["p50_ms"] / row["continuous"]["p50_ms"]
        row["p99_ratio"] = row["serial"]["p99_ms"] / row["continuous"]["p99_ms"]
        out[f"rate_{int(rate)}"] = row
    srv.close()
    return out


def _gemm_step_fn(g, A, B, C, M, N, K, engine, ws):
    def step():
        g.matmul(A, B, M, N, K, C=C, engine=engine, workspace=ws)
    return step


def run_ours(args, rank, world, local):
    import torch

    import gatlas_b200 as g

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    peaks = _peaks()
    engine = HEADLINE_ENGINE if g.matmul_supported(HEADLINE_ENGINE) else "buffer"

    # ---- headline: FP32-accurate SGEMM 8192^3 --------------------------------
    M = N = K = M_GEMM
    A = torch.empty(M * K, dtype=torch.float32, device=dev)
    B = torch.empty(K * N, dtype=torch.float32, device=dev)
    C = torch.empty(M * N, dtype=torch.float32, device=dev)
    g.fill(A, "uniform", seed=1 + rank)
    g.fill(B, "uniform", seed=2 + rank)
    ws_bytes = max(g.matmul_workspace_size(M, N, K, e) for e in SWEEP_ENGINES if e != "buffer")
    ws = torch.empty(ws_bytes + 1024, dtype=torch.uint8, device=dev)
    ws = ws[(-ws.data_ptr()) % 1024:][:ws_bytes]          # 1024-byte aligned view
    step = _gemm_step_fn(g, A, B, C, M, N, K, engine, ws if engine != "buffer" else None)
    launches_per_step = 1 if engine == "buffer" else 3     # split A, split B, contraction

    sampler = ClockSampler(local)
    ms = _timed(step, args.steps, args.warmup, world, stream, sampler=sampler)
    clocks = sampler.clocks
    flops = 2.0 * M * N * K
    value, ms_max = _aggregate(flops, ms, world)
    fro, refn, mx, _ = g.residual(A, B, C, M, N, K)

    # dominant kernel alone: the tcgen05 contraction on prepared operands
    if engine != "buffer":
        g.matmul_tc_prepare(A, B, M, N, K, ws, engine=engine)
        run_ms = _timed(lambda: g.matmul_tc_run(ws, M, N, K, C, engine=engine), args.steps, 2,
                        world, stream)
        ach = PRODUCTS[engine] * flops / (run_ms * 1e-3) / 1e12
        roofline = {"bound": "tensor", "kernel": TC_KERNEL, "achieved": ach,
                    "peak": peaks["bf16_tflops"], "unit": "TFLOP/s",
                    "frac": ach / peaks["bf16_tflops"], "traffic": TC_TRAFFIC_BYTES,
                    "kernel_ms": run_ms, "kernel_fp32_equiv_tflops": flops / (run_ms * 1e-3) / 1e12,
                    "peak_source": f"{peaks['source']} dense BF16 (burst, cuBLAS); achieved counts all "
                                   f"{PRODUCTS[engine]} BF16 products per FP32 multiply-add; 'of measured'",
                    "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per launch, "
                                      "profiles/tc_gemm_persistent_split3_pair_8192.md"}
    else:
        roofline = {"bound": "fp32_simt", "achieved": value, "peak": FP32_SIMT_NOMINAL_TFLOPS,
                    "unit": "TFLOP/s", "frac": value / FP32_SIMT_NOMINAL_TFLOPS, "traffic": None,
                    "peak_source": "nominal (148 SMs x 128 lanes x 2 x 1.965 GHz)"}

    # ---- e2e through the C ABI with host buffers ------------------------------
    hA = torch.empty(M * K, dtype=torch.float32, pin_memory=True)
    hB = torch.empty(K * N, dtype=torch.float32, pin_memory=True)
    hC = torch.empty(M * N, dtype=torch.float32, pin_memory=True)
    hA.copy_(A)
    hB.copy_(B)

    def e2e_step():
        # one public call with host buffers: uploads, contraction and download,
        # pipelined over row blocks of A by the library
        g.matmul_host(hA, hB, M, N, K, hC, engine=engine)

    e2e_ms = _max_over_ranks(_timed(e2e_step, max(2, min(args.steps, 10)), 1, world, stream), world)
    e2e = {"value": world * flops / (e2e_ms * 1e-3) / 1e12, "unit": "TFLOP/s",
           "h2d_bytes_per_step": 2 * M * K * 4, "d2h_bytes_per_step": M * N * 4,
           "ms_per_step": e2e_ms,
           "path": "gatlas_matmul_f32_host: pinned host A, B in, C out (B uploaded and split once, A in "
                   "512-row blocks whose uploads, splits, contraction and C downloads overlap on three streams)"}
    del hA, hB, hC

    # ---- precision sweep (8192^3; DGEMM 4096^3) -------------------------------
    sweep = {}
    if not args.quick:
        for dist in ("uniform", "pow2"):
            g.fill(A, dist, seed=11)
            g.fill(B, dist, seed=12)
            for eng in SWEEP_ENGINES:
                if not g.matmul_supported(eng):
                    continue
                f = _gemm_step_fn(g, A, B, C, M, N, K, eng, ws if eng != "buffer" else None)
                t = _timed(f, 3 if eng == "buffer" else 5, 1, world, stream)
                fr, rn, mxe, _ = g.residual(A, B, C, M, N, K)
                row = {"tflops": flops / (t * 1e-3) / 1e12, "ms": t, "normwise_err": fr / rn,
                       "max_abs_err": mxe}
                if eng != "buffer":
                    # the contraction alone on operands prepared once
                    g.matmul_tc_prepare(A, B, M, N, K, ws, engine=eng)
                    tk = _timed(lambda: g.matmul_tc_run(ws, M, N, K, C, engine=eng), 5, 1, world, stream)
                    row["kernel_ms"] = tk
                    row["kernel_tflops"] = flops / (tk * 1e-3) / 1e12
                sweep[f"{eng}_{dist}"] = row
        Md = 4096
        Ad = torch.empty(Md * Md, dtype=torch.float64, device=dev)
        Bd = torch.empty(Md * Md, dtype=torch.float64, device=dev)
        Cd = torch.empty(Md * Md, dtype=torch.float64, device=dev)
        g.fill(Ad, "uniform", seed=13)
        g.fill(Bd, "uniform", seed=14)
        t = _timed(lambda: g.matmul(Ad, Bd, Md, Md, Md, C=Cd), 3, 1, world, stream)
        sweep["dgemm_buffer_4096"] = {"tflops": 2.0 * Md ** 3 / (t * 1e-3) / 1e12, "ms": t}
        del Ad, Bd, Cd
    del C, ws

    # ---- memory-bound pair: GEMV 16384^2, SAXPY 2^28
    secondary = {}
    Ag = torch.empty(N_GEMV * N_GEMV, dtype=torch.float32, device=dev)
    xg = torch.empty(N_GEMV, dtype=torch.float32, device=dev)
    yg = torch.empty(N_GEMV, dtype=torch.float32, device=dev)
    g.fill(Ag, "uniform", seed=3)
    g.fill(xg, "uniform", seed=4)
    gemv_bytes = 4.0 * (N_GEMV * N_GEMV + 2 * N_GEMV)
    for ta in (0, 1):
        for eng in ("buffer", "image"):
            try:
                g.matvec(Ag, xg, N_GEMV, N_GEMV, y=yg, trans_a=ta, engine=eng)
            except g.GatlasError:
                continue
            t = _timed(lambda: g.matvec(Ag, xg, N_GEMV, N_GEMV, y=yg, trans_a=ta, engine=eng),
                       max(args.steps, 10), 3, world, stream)
            secondary[f"sgemv_{'At' if ta else 'A'}x_{eng}_gbs"] = gemv_bytes / (t * 1e-3) / 1e9
    del Ag, xg, yg
    xs = torch.empty(N_SAXPY, dtype=torch.float32, device=dev)
    ys = torch.empty(N_SAXPY, dtype=torch.float32, device=dev)
    g.fill(xs, "uniform", seed=5)
    g.fill(ys, "uniform", seed=6)
    for eng in ("buffer", "image"):
        t = _timed(lambda: g.saxpy(0.5, xs, ys, out=ys, engine=eng), max(args.steps, 10), 3,
                   world, stream)
        secondary[f"saxpy_{eng}_gbs"] = 12.0 * N_SAXPY / (t * 1e-3) / 1e9
    for k in [k for k in secondary if k.endswith("_gbs")]:
        secondary[k.replace("_gbs", "_hbm_frac")] = secondary[k] / peaks["hbm_gbs"]
    secondary["hbm_peak_gbs"] = peaks["hbm_gbs"]
    del xs, ys

    # ---- plain SGEMM 1024^3, autotuned SIMT point ---------------------------------
    sgemm_1024 = sgemm_autotune_leg(world, stream)

    # ---- batched uneven GEMM (grouped persistent kernel) ------------------------
    grouped = grouped_leg(args, world, stream) if not args.quick else None

    # ---- serving stream (continuous batching vs serial) -------------------------
    serving = serving_leg(args) if not args.quick else None

    faults = g.device_faults()
    cpu = cpu_baseline(args.cpu_seconds) if (rank == 0 and world == 1 and not args.no_cpu) else None

    # the memory-bound kernels against measured HBM bandwidth (same roofline
    # terms as the headline kernel: algorithmic bytes / event time)
    others = []
    for key, kern in (("sgemv_Ax_buffer_gbs", "gemv_rowblock_kernel"), ("sgemv_Atx_buffer_gbs", "gemv_cols_kernel"),
                      ("sgemv_Ax_image_gbs", "gemv_rows_tma_kernel"), ("sgemv_Atx_image_gbs", "gemv_cols_tma_kernel"),
                      ("saxpy_buffer_gbs", "saxpy_vec_kernel"), ("saxpy_image_gbs", "saxpy_bulk_kernel")):
        if key in secondary:
            others.append({"kernel": kern, "workload": key[:-4], "bound": "hbm", "achieved": round(secondary[key], 1),
                           "peak": peaks["hbm_gbs"], "unit": "GB/s",
                           "frac": round(secondary[key] / peaks["hbm_gbs"], 3)})
    # the grouped contraction (graph of the contraction alone, operands
    # resident): every BF16 product's FLOPs against the measured BF16 peak
    for eng in ("tc_split3", "tc_bf16"):
        row = (grouped or {}).get(eng)
        if row:
            ach = PRODUCTS[eng] * row["tflops_graph_run"]
            others.append({"kernel": f"grouped_gemm_kernel<{eng[3:]}>", "workload": "grouped_1024", "bound": "tensor",
                           "achieved": round(ach, 1), "peak": peaks["bf16_tflops"], "unit": "TFLOP/s",
                           "frac": round(ach / peaks["bf16_tflops"], 3)})
    roofline["others"] = others
    target = _target(sweep, value, fro / refn)

    out = {
        "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded uniform[-1,1) FP32 operands generated on the device)",
        "config": {"workload": "sgemm_fp32_accurate_8192", "m": M, "n": N, "k": K,
                   "engine": engine, "layout": "row-major, no transposes",
                   "step": "split A and B into BF16 pieces + tcgen05 contraction (one "
                           "gatlas_matmul_f32 call)",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2": "operands larger than L2; no flush"},
        "error_vs_fp64": {"normwise": fro / refn, "max_abs": mx},
        "e2e": e2e, "roofline": roofline, "precision_sweep": sweep, "secondary": secondary,
        "sgemm_1024_autotune": sgemm_1024, "grouped": grouped, "serving": serving,
        "gpu_launches": launches_per_step * args.steps, "clocks": clocks,
        "device_faults": faults,
    }
    if cpu:
        out["cpu_baseline"] = cpu
    out["target"] = target
    # last key, so that a reader of only the end of the line sees every leg
    out["summary"] = _summary(out)
    return out


def _target(sweep: dict, headline_tflops: float, headline_err: float) -> dict:
    """The precision target at 8192^3: the split-BF16 engines against the
    plain SIMT FP32 kernel, >= 3x its TFLOP/s at equal or better normwise
    error against the FP64 product (uniform operands)."""
    simt = sweep.get("buffer_uniform")
    if not simt:
        return {}
    out = {"simt_fp32": {"tflops": round(simt["tflops"], 2), "err": simt["normwise_err"]}}
    for eng in ("tc_split3", "tc_split6"):
        row = sweep.get(f"{eng}_uniform")
        if not row:
            continue
        ratio = row["tflops"] / simt["tflops"]
        out[eng] = {"tflops": round(row["tflops"], 1), "err": row["normwise_err"], "x_simt": round(ratio, 2),
                    "meets": bool(ratio >= 3.0 and row["normwise_err"] <= simt["normwise_err"])}
    return out


def _summary(o: dict) -> dict:
    """One compact object with every leg's figures."""
    r = lambda v, n=1: None if v is None else round(v, n)
    sec = o.get("secondary") or {}
    sm = {"headline_tflops": r(o["value"]), "e2e_tflops": r(o["e2e"]["value"]),
          "tc_frac": r(o["roofline"].get("frac"), 3), "err": o.get("error_vs_fp64", {}).get("normwise")}
    sm["hbm_frac"] = {k[:-9]: r(v, 3) for k, v in sec.items() if k.endswith("_hbm_frac")}
    sw = o.get("precision_sweep") or {}
    sm["sweep_kernel_tflops"] = {k.replace("_uniform", ""): r(v.get("kernel_tflops", v["tflops"]))
                                 for k, v in sw.items() if not k.endswith("_pow2")}
    sm["target"] = o.get("target")
    a = o.get("sgemm_1024_autotune") or {}
    if a:
        sm["sgemm_1024"] = {"tflops": r(a["best_tflops"], 2), "tile": list(a["best_tile"].values()),
                            "err": a["error_vs_fp64"]["normwise"]}
    gr = o.get("grouped") or {}
    sm["grouped"] = {e: {"x_per_instance": r(gr[e]["speedup_vs_per_instance"], 2),
                         "tflops_run": r(gr[e]["tflops_graph_run"])} for e in ("tc_split3", "tc_bf16") if e in gr}
    sv = o.get("serving") or {}
    sm["serving"] = {k: {"rps": [r(v["continuous"]["throughput_rps"], 0), r(v["serial"]["throughput_rps"], 0)],
                         "p99_ms": [r(v["continuous"]["p99_ms"], 2), r(v["serial"]["p99_ms"], 2)]}
                     for k, v in sv.items() if k.startswith("rate_")}
    cb = o.get("cpu_baseline") or {}
    if cb:
        sm["cpu"] = {"tflops": r(cb["value"], 4), "kind": cb["kind"], "cores": cb["cores"],
                     "secondary": {k: float(f"{v:.4g}") for k, v in (cb.get("secondary") or {}).items()}}
    return sm


# ---------------------------------------------------------------------------
# CPU legs: the reference's own generated kernels on the host cores
# ---------------------------------------------------------------------------
#
# oracle/_ref holds the reference's buffer matmul, matvec and saxpy kernels,
# emitted by the reference's generators and compiled for the host CPU (mad
# fused); they run one work group per core at a time (OpenMP over work
# groups).  Where that library is absent the oracle's port of the buffer
# kernel's algorithm stands in (kind "port").

REF_SGEMM = "bench_sgemm_8192"    # float4, 16 x 16 work items, 8 x 4 inner blocking, extra 0


def _ref_kernels():
    try:
        import oracle.ref as R
        return R if R.available() else None
    except Exception:
        return None


def _ref_band_rows(R) -> int:
    k = R.kernel(REF_SGEMM)
    return k["local"][1] * k["params"][9]   # work-group height x inner blocking height


def _ref_sgemm_sample(R, seconds: float, threads: int):
    """Bands of work groups (128 rows of C each) of the reference's 8192^3
    buffer kernel that take about `seconds` on the host cores: (A, B, C,
    bands); A holds only the sampled rows."""
    import numpy as np

    import oracle
    K = N = M_GEMM
    rows = _ref_band_rows(R)
    B = oracle.uniform(K * N, seed=2)
    A = oracle.uniform(rows * K, seed=1)
    Afull = np.zeros(M_GEMM * K, np.float32)   # kernel reads A through its band offset
    Afull[: rows * K] = A
    C = np.zeros(M_GEMM * N, np.float32)
    t0 = time.perf_counter()
    R.run(REF_SGEMM, Afull, B, C, group_begin=(0, 0), group_end=(0, 1), threads=threads)
    dt = max(time.perf_counter() - t0, 1e-3)
    bands = max(1, min(M_GEMM // rows, int(seconds / dt)))
    Afull[: bands * rows * K] = oracle.uniform(bands * rows * K, seed=1)
    return Afull, B, C, bands


def _ref_secondary(R, threads: int) -> dict:
    """The reference's memory-bound kernels at the workload sizes (SAXPY
    n = 2^28 as 2^26 float4; SGEMV 16384^2, both layouts, buffer and image)
    and its SGEMM 1024^3 point, timed once each after one untimed call; and
    the naive host loop at 1024^3 on one thread."""
    import numpy as np

    import oracle
    out = {}
    n = N_SAXPY
    X, Y = oracle.uniform(n, seed=5), oracle.uniform(n, seed=6)
    Z = np.empty_like(X)
    R.run("bench_saxpy_2p28", X, Y, Z, 0.5, threads=threads)
    t0 = time.perf_counter()
    R.run("bench_saxpy_2p28", X, Y, Z, 0.5, threads=threads)
    out["saxpy_gbs"] = 12.0 * n / (time.perf_counter() - t0) / 1e9
    del X, Y, Z
    Ag, xg = oracle.uniform(N_GEMV * N_GEMV, seed=3), oracle.uniform(N_GEMV, seed=4)
    yg = np.zeros(N_GEMV, np.float32)
    for kid, key in (("bench_sgemv_n_16384", "sgemv_Ax_buffer_gbs"), ("bench_sgemv_t_16384", "sgemv_Atx_buffer_gbs"),
                     ("bench_sgemv_img_n_16384", "sgemv_Ax_image_gbs"),
                     ("bench_sgemv_img_t_16384", "sgemv_Atx_image_gbs")):
        R.run(kid, Ag, xg, yg, threads=threads)
        t0 = time.perf_counter()
        R.run(kid, Ag, xg, yg, threads=threads)
        out[key] = 4.0 * (N_GEMV * N_GEMV + 2 * N_GEMV) / (time.perf_counter() - t0) / 1e9
    del Ag, xg, yg
    m = SGEMM_TUNE_N
    A1, B1, C1 = oracle.uniform(m * m, seed=1), oracle.uniform(m * m, seed=2), np.zeros(m * m, np.float32)
    R.run("bench_sgemm_1024", A1, B1, C1, threads=threads)
    t0 = time.perf_counter()
    R.run("bench_sgemm_1024", A1, B1, C1, threads=threads)
    out["sgemm_1024_tflops"] = 2.0 * m ** 3 / (time.perf_counter() - t0) / 1e12
    # the reference's naive host check loop (KernelMatmulBuffer.hpp:124-143,
    # restated in the oracle), one thread as the reference runs it
    t0 = time.perf_counter()
    oracle.matmul(A1, B1, m, m, m, mode=oracle.REFHOST, threads=1)
    out["sgemm_1024_host_loop_tflops"] = 2.0 * m ** 3 / (time.perf_counter() - t0) / 1e12
    return out


def _cpu_rows_for(seconds: float, threads: int) -> int:
    """Rows of C whose computation takes about `seconds` on the host cores
    (from a 16-row pilot), a multiple of 16 in [16, 8192] (oracle port)."""
    import oracle
    K = N = M_GEMM
    A = oracle.uniform(16 * K, seed=1)
    B = oracle.uniform(K * N, seed=2)
    t0 = time.perf_counter()
    oracle.matmul_tiled(A, B, 16, N, K, tile_m=16, tile_n=64, threads=threads)
    dt = max(time.perf_counter() - t0, 1e-3)
    rows = int(16 * seconds / dt) // 16 * 16
    return max(16, min(M_GEMM, rows))


def cpu_baseline(seconds: float) -> dict:
    """The reference's 8192^3 buffer kernel on the host cores, on a bounded
    sample of the workload: the first bands of work groups, sized to about
    `seconds` of CPU work; plus the reference's memory-bound kernels and its
    SGEMM 1024^3 point."""
    import oracle
    threads = oracle.max_threads()
    K = N = M_GEMM
    R = _ref_kernels()
    if R is not None:
        A, B, C, bands = _ref_sgemm_sample(R, seconds, threads)
        rows = bands * _ref_band_rows(R)
        t0 = time.perf_counter()
        R.run(REF_SGEMM, A, B, C, group_begin=(0, 0), group_end=(0, bands), threads=threads)
        dt = time.perf_counter() - t0
        del A, B, C
        flops = 2.0 * rows * N * K
        return {"value": flops / dt / 1e12, "unit": "TFLOP/s", "cores": threads, "kind": "reference",
                "sample": f"{rows} of 8192 rows of C ({bands} bands of work groups) of the reference's "
                          f"matmulbufferfloat4 (16x16 work items, 8x4 blocking) at 8192^3: "
                          f"{flops / 1e9:.0f} GFLOP in {dt:.1f} s",
                "kernels": "oracle/_ref: the reference's emitted OpenCL C compiled for the host, mad fused",
                "secondary": _ref_secondary(R, threads)}
    rows = _cpu_rows_for(seconds, threads)
    A = oracle.uniform(rows * K, seed=1)
    B = oracle.uniform(K * N, seed=2)
    t0 = time.perf_counter()
    oracle.matmul_tiled(A, B, rows, N, K, tile_m=128, tile_n=64, threads=threads)
    dt = time.perf_counter() - t0
    flops = 2.0 * rows * N * K
    return {"value": flops / dt / 1e12, "unit": "TFLOP/s", "cores": threads, "kind": "port",
            "sample": f"{rows} of 8192 rows of C of the 8192^3 SGEMM "
                      f"({flops / 1e9:.0f} GFLOP in {dt:.1f} s)"}


def run_reference(args, rank, world):
    if rank != 0:
        return None
    import oracle
    threads = oracle.max_threads()
    K = N = M_GEMM
    # each step a bounded sample sized so the whole run takes a few minutes
    per_step_s = max(1.0, min(8.0, 150.0 / max(1, args.steps + args.warmup)))
    R = _ref_kernels()
    if R is not None:
        A, B, C, bands = _ref_sgemm_sample(R, per_step_s, threads)
        rows = bands * _ref_band_rows(R)
        step = lambda: R.run(REF_SGEMM, A, B, C, group_begin=(0, 0), group_end=(0, bands), threads=threads)
        kind = "reference"
        engine = ("the reference's matmulbufferfloat4 kernel (emitted by its generator, 16x16 work items, "
                  "8x4 blocking) compiled for the host cores, mad fused (oracle/_ref)")
        sample = f"{rows} of 8192 rows of C ({bands} bands of work groups) of the 8192^3 SGEMM per step"
    else:
        rows = _cpu_rows_for(per_step_s, threads)
        A = oracle.uniform(rows * K, seed=1)
        B = oracle.uniform(K * N, seed=2)
        step = lambda: oracle.matmul_tiled(A, B, rows, N, K, tile_m=128, tile_n=64, threads=threads)
        kind = "port"
        engine = "the reference's buffer-kernel algorithm on the host cores (oracle port)"
        sample = f"{rows} of 8192 rows of C of the 8192^3 SGEMM per step"
    for _ in range(min(args.warmup, 1)):
        step()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        step()
        times.append(time.perf_counter() - t0)
    dt = sum(times) / len(times)
    flops = 2.0 * rows * N * K
    v = flops / dt / 1e12
    return {
        "metric": METRIC, "value": v, "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "impl": "reference",
        "data": "synthetic (seeded uniform[-1,1) FP32 operands)",
        "config": {"workload": "sgemm_fp32_accurate_8192", "m": M_GEMM, "n": M_GEMM, "k": M_GEMM,
                   "engine": engine},
        "cpu_baseline": {"value": v, "unit": "TFLOP/s", "cores": threads, "kind": kind, "sample": sample},
        "e2e": {"value": v, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def run_case(spec: str) -> None:
    """Small single-kernel cases for ncu captures: NAME:SIZE, three calls each.
    tc_bf16|tc_split3|tc_split6|tc_fp8[_pair]:M (M^3 GEMM, prepare once, run x3; _pair forces CTA pairs),
    sgemm_simt:M, sgemm_image:M, dgemm_simt:M (M^3 float64 on the SIMT engine),
    quant_fp8:M (the FP8 operand pass, x3), split3_prepare:M (the split-BF16 operand pass, x3),
    gemv_A:N / gemv_At:N (N^2 GEMV, buffer engine), gemv_img_A:N / gemv_img_At:N (TMA engine),
    dgemv_A:N / dgemv_At:N / dgemv_img_A:N / dgemv_img_At:N (float64), saxpy_buffer:n / saxpy_image:n,
    grouped_tc_split3|grouped_tc_bf16:count (the batched workload)."""
    import torch

    import gatlas_b200 as g
    name, size = spec.split(":")
    size = int(size)
    if name.endswith("_pair"):  # the same case on CTA pairs (cta_group::2)
        name = name[:-len("_pair")]
        import gatlas_b200 as gb
        gb.set_option("tc_pair", 2)
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    if name == "dgemm_simt":
        M = size
        A = torch.empty(M * M, dtype=torch.float64, device=dev)
        B = torch.empty(M * M, dtype=torch.float64, device=dev)
        C = torch.empty(M * M, dtype=torch.float64, device=dev)
        g.fill(A, "uniform", seed=1)
        g.fill(B, "uniform", seed=2)
        for _ in range(3):
            g.matmul(A, B, M, M, M, C=C)
    elif name == "split3_prepare":
        M = size
        A = torch.empty(M * M, device=dev)
        B = torch.empty(M * M, device=dev)
        g.fill(A, "uniform", seed=1)
        g.fill(B, "uniform", seed=2)
        ws = torch.empty(g.matmul_workspace_size(M, M, M, "tc_split3") + 1024, dtype=torch.uint8, device=dev)
        ws = ws[(-ws.data_ptr()) % 1024:]
        for _ in range(3):
            g.matmul_tc_prepare(A, B, M, M, M, ws, engine="tc_split3")
    elif name.startswith("tc_") or name in ("sgemm_simt", "sgemm_image", "quant_fp8"):
        M = size
        A = torch.empty(M * M, device=dev)
        B = torch.empty(M * M, device=dev)
        C = torch.empty(M * M, device=dev)
        g.fill(A, "uniform", seed=1)
        g.fill(B, "uniform", seed=2)
        if name == "sgemm_simt":
            for _ in range(3):
                g.matmul(A, B, M, M, M, C=C)
        elif name == "sgemm_image":
            for _ in range(3):
                g.matmul(A, B, M, M, M, C=C, engine="image")
        elif name == "quant_fp8":
            ws = torch.empty(g.matmul_workspace_size(M, M, M, "tc_fp8") + 1024, dtype=torch.uint8, device=dev)
            ws = ws[(-ws.data_ptr()) % 1024:]
            for _ in range(3):
                g.matmul_tc_prepare(A, B, M, M, M, ws, engine="tc_fp8")
        else:
            ws = torch.empty(g.matmul_workspace_size(M, M, M, name) + 1024, dtype=torch.uint8, device=dev)
            ws = ws[(-ws.data_ptr()) % 1024:]
            g.matmul_tc_prepare(A, B, M, M, M, ws, engine=name)
            for _ in range(3):
                g.matmul_tc_run(ws, M, M, M, C, engine=name)
    elif name.startswith("gemv_") or name.startswith("dgemv_"):
        N = size
        dt = torch.float64 if name.startswith("d") else torch.float32
        A = torch.empty(N * N, dtype=dt, device=dev)
        x = torch.empty(N, dtype=dt, device=dev)
        y = torch.empty(N, dtype=dt, device=dev)
        g.fill(A, "uniform", seed=1)
        g.fill(x, "uniform", seed=2)
        eng = "image" if "_img_" in name else "buffer"
        for _ in range(3):
            g.matvec(A, x, N, N, y=y, trans_a=name.endswith("_At"), engine=eng)
    elif name.startswith("saxpy_"):
        x = torch.empty(size, device=dev)
        y = torch.empty(size, device=dev)
        g.fill(x, "uniform", seed=1)
        g.fill(y, "uniform", seed=2)
        for _ in range(3):
            g.saxpy(0.5, x, y, out=y, engine=name.split("_")[1])
    elif name.startswith("grouped_"):
        # the batched workload with `size` instances, contraction launched x3
        inst, bufs = grouped_workload(dev, count=size)
        plan = g.Grouped(inst, engine=name.split("_", 1)[1])
        plan.prepare()
        for _ in range(3):
            plan.run()
    else:
        raise SystemExit(f"unknown case {spec}")
    torch.cuda.synchronize()
    print(json.dumps({"case": spec, "faults": g.device_faults()}))


def run_tc_sweep(args) -> None:
    """Sustained timing of the tensor-core contraction on prepared operands:
    per size, engine, CTA-pair setting (0 single, 2 pairs) and raster group
    height, about `--sweep-seconds` of back-to-back launches with the SM clock
    sampled through NVML.  One JSON line per point; cycles = ms x median MHz.
    Pair settings (gatlas_set_option "tc_pair"): 1 the default choice (CTA
    pairs for split3/split6, 256 x 256 single-CTA tiles for BF16), 0 single
    CTAs on 128 x 256 tiles, 2 CTA pairs.  L2 hint ("tc_l2_hint"): 1 (the
    default) A's loads evict-last, 0 none."""
    import time

    import torch

    import gatlas_b200 as g
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    engines = args.sweep_engines.split(",")
    rows_list = [int(x) for x in args.sweep_group_rows.split(",")]
    hints = [int(x) for x in args.sweep_l2_hints.split(",")]
    for M in (int(x) for x in args.tc_sweep.split(",")):
        A = torch.empty(M * M, device=dev)
        B = torch.empty(M * M, device=dev)
        C = torch.empty(M * M, device=dev)
        g.fill(A, "uniform", seed=1)
        g.fill(B, "uniform", seed=2)
        for eng in engines:
            for pair in (int(x) for x in args.sweep_pairs.split(",")):
                g.set_option("tc_pair", pair)
                ws = torch.empty(g.matmul_workspace_size(M, M, M, eng) + 1024, dtype=torch.uint8, device=dev)
                ws = ws[(-ws.data_ptr()) % 1024:]
                g.matmul_tc_prepare(A, B, M, M, M, ws, engine=eng)
                for rows, hint in ((r, h) for r in rows_list for h in hints):
                    g.set_option("tc_group_rows", rows)
                    g.set_option("tc_l2_hint", hint)
                    for _ in range(3):
                        g.matmul_tc_run(ws, M, M, M, C, engine=eng)
                    torch.cuda.synchronize()
                    t0 = time.perf_counter()
                    g.matmul_tc_run(ws, M, M, M, C, engine=eng)
                    torch.cuda.synchronize()
                    n = max(10, int(args.sweep_seconds / max(time.perf_counter() - t0, 1e-6)))
                    sampler = ClockSampler(0)
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    sampler.start()
                    e0.record()
                    for _ in range(n):
                        g.matmul_tc_run(ws, M, M, M, C, engine=eng)
                    e1.record()
                    torch.cuda.synchronize()
                    clocks = sampler.stop()
                    ms = e0.elapsed_time(e1) / n
                    mhz = clocks.get("sm_mhz")
                    work = PRODUCTS.get(eng, 1) * 2.0 * M ** 3
                    print(json.dumps({"m": M, "engine": eng, "pair": pair, "group_rows": rows, "l2_hint": hint,
                                      "launches": n,
                                      "ms": round(ms, 4), "tflops_fp32_work": round(2.0 * M ** 3 / ms / 1e9, 1),
                                      "tflops_tensor_work": round(work / ms / 1e9, 1), "sm_mhz": mhz,
                                      "mcycles": round(ms * mhz / 1e3, 3) if mhz else None,
                                      "reasons": clocks.get("reasons"), "faults": g.device_faults()}), flush=True)
                del ws
                torch.cuda.empty_cache()
    g.set_option("tc_pair", 1)
    g.set_option("tc_group_rows", 2048)
    g.set_option("tc_l2_hint", 1)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="CPU work in the cpu_baseline sample")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--quick", action="store_true", help="skip the precision sweep")
    ap.add_argument("--case", default=None, help="run one small single-kernel case (for ncu) and exit")
    ap.add_argument("--tc-sweep", default=None,
                    help="sizes (comma-separated): sustained timing of the tensor-core contraction on single CTAs "
                         "and CTA pairs, with SM clocks, one JSON line per point, then exit")
    ap.add_argument("--sweep-engines", default="tc_bf16,tc_split3,tc_split6")
    ap.add_argument("--sweep-group-rows", default="2048", help="raster group heights to sweep (multiples of 128)")
    ap.add_argument("--sweep-seconds", type=float, default=1.5)
    ap.add_argument("--sweep-pairs", default="1,0,2", help="tc_pair settings to sweep")
    ap.add_argument("--sweep-l2-hints", default="1", help="tc_l2_hint settings to sweep")
    ap.add_argument("--option", action="append", default=[], metavar="NAME=VALUE",
                    help="gatlas_set_option before a --case or --tc-sweep run (repeatable)")
    args = ap.parse_args()
    if args.option:
        import gatlas_b200 as g
        for o in args.option:
            name, value = o.split("=", 1)
            g.set_option(name, int(value))
    if args.tc_sweep:
        run_tc_sweep(args)
        return
    if args.case:
        run_case(args.case)
        return
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.impl == "reference":
        res = run_reference(args, rank, world)
        if res is not None:
            print(json.dumps(res), flush=True)
        return
    rank, world, local = _dist_init(args.gpus)
    res = run_ours(args, rank, world, local)
    if rank == 0:
        print(json.dumps(res), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
