"""Command-line tools on CPU: print_*, purgeJournal, a journal-replayed search
(no device touched) and retry.  Crash/resume is exercised by journals whose
last record for a key is BUILD_IN_PROGRESS or RUN_IN_PROGRESS -- what a
process killed while building or running a point leaves behind."""
import os
import subprocess

import pytest

from gatlas_b200.plugin import Kernel
from oracle.params import BUILD_IN_PROGRESS, BUILD_OK, RUN_IN_PROGRESS, RUN_OK, Journal, journal_key

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "gatlas_b200", "bin")


def run(args, **kw):
    return subprocess.run([os.path.join(BIN, args[0])] + args[1:], capture_output=True, text=True,
                          timeout=120, **kw)


def test_print_matmul_valid_and_invalid():
    r = run(["print_matmul", "-T", "floatimg", "-G", "-n", "3520", "-g", "8", "-y", "8", "-x", "1"])
    assert r.returncode == 0
    assert "matmulimagefloat4" in r.stdout and "extra parameter 1 = (1 0 0)" in r.stdout
    r = run(["print_matmul", "-T", "float4", "-n", "100", "-g", "16", "-y", "8", "-x", "0"])
    assert r.returncode == 1 and "invalid parameters" in r.stderr
    r = run(["print_matmul", "-T", "float4", "-n", "1024", "-g", "17", "-y", "8", "-x", "0"])
    assert r.returncode == 1 and "from 1 to 16" in r.stderr
    r = run(["print_matvec", "-T", "float4", "-n", "16384", "-g", "64", "-y", "4", "-x", "1", "-a"])
    assert r.returncode == 0 and "matvecbufferfloat4" in r.stdout
    r = run(["print_saxpy", "-T", "float4", "-m", "67108864", "-Y", "256", "-y", "4", "-x", "0"])
    assert r.returncode == 0 and "saxpybufferfloat4" in r.stdout


def test_purge_journal_matches_reference_semantics(tmp_path):
    lines = [
        ("k_good_", RUN_IN_PROGRESS), ("k_good_", RUN_OK), ("k_good_", 120), ("k_good_", 118),
        ("k_crash_build_", BUILD_IN_PROGRESS),
        ("k_hang_", BUILD_IN_PROGRESS), ("k_hang_", BUILD_OK), ("k_hang_", RUN_IN_PROGRESS),
        ("k_failed_", RUN_OK), ("k_failed_", 0),
        ("a_first_", RUN_OK), ("a_first_", 55),
    ]
    text = "".join(f"{k}\t{v}\n" for k, v in lines)
    for delete in (False, True):
        p1 = tmp_path / f"ours_{delete}.journal"
        p2 = tmp_path / f"oracle_{delete}.journal"
        p1.write_text(text)
        p2.write_text(text)
        args = ["purgeJournal", "-j", str(p1)] + (["-d"] if delete else [])
        r = run(args)
        assert r.returncode == 0
        j = Journal(str(p2))
        assert j.load()
        good = len(j.times)
        bad = j.purge(delete)
        assert r.stdout.strip() == (f"journal file {p1} has {bad} bad keys, "
                                    f"{'deleted' if delete else 'preserved'} {good} good keys")
        assert p1.read_text() == p2.read_text()
    assert bad == 2  # crashed while building, hung while running


def _points(n, g, bh, vl=4):
    k = Kernel("matmul", "float4")
    pts = []
    for x in range(12):
        p = [1, 0, n, n, n, 0, 0, g, g, bh, vl, x]
        k.set_params(p)
        ok, q = k.get_params()
        assert ok
        pts.append(q)
    return k, pts


def test_search_replays_journal_without_a_device(tmp_path):
    k, pts = _points(256, 16, 8)
    name = k.kernel_name()
    # x = 0..7 ran (two trials each), 8 failed its check, 9 crashed while
    # building, 10 hung while running, 11 had its build fail
    j = tmp_path / "replay.journal"
    recs = []
    times = {}
    for x, p in enumerate(pts):
        key = journal_key(name, p)
        if x < 8:
            t = [100 + 7 * x, 101 + 7 * x]
            times[x] = t
            recs += [(key, BUILD_IN_PROGRESS), (key, BUILD_OK), (key, RUN_IN_PROGRESS), (key, RUN_OK),
                     (key, t[0]), (key, RUN_OK), (key, t[1])]
        elif x == 8:
            recs += [(key, RUN_OK), (key, 0)]
        elif x == 9:
            recs += [(key, BUILD_IN_PROGRESS)]
        elif x == 10:
            recs += [(key, BUILD_OK), (key, RUN_IN_PROGRESS)]
        else:
            recs += [(key, BUILD_IN_PROGRESS)]
    j.write_text("".join(f"{a}\t{b}\n" for a, b in recs))
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = run(["bench_matmul", "-d", "gpu0", "-j", str(j), "-T", "float4", "-n", "256", "-g", "16", "-y", "8",
             "-t", "2"], env=env)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip().endswith("***DONE***")
    assert r.stdout.count("bad") >= 3 * 2 - 3   # crashed/hung points reported as bad
    final = [ln for ln in r.stdout.splitlines() if ln.startswith("[") and " usec\tavg: " in ln]
    assert len(final) == 8
    # fastest accumulated time first; avg = flops/usec/1000 averaged over the trials (Welford)
    flops = 256 * 256 * (2 * 256 - 1)
    for rank, ln in enumerate(final):
        x = rank
        accum = sum(times[x])
        assert ln.startswith(f"[{rank}] {accum} usec\tavg: ")
        avg = float(ln.split("avg: ")[1].split("\t")[0])
        want = (flops / times[x][0] / 1000 + flops / times[x][1] / 1000) / 2
        assert avg == pytest.approx(want, rel=1e-5)
        assert ln.rstrip().endswith(f"({x % 2} {x // 2})")
    # the journal is unchanged: nothing ran
    assert j.read_text() == "".join(f"{a}\t{b}\n" for a, b in recs)


def test_search_without_device_refuses_unrecorded_points(tmp_path):
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    j = tmp_path / "empty.journal"
    r = run(["bench_matmul", "-d", "gpu0", "-j", str(j), "-T", "float4", "-n", "256", "-g", "16", "-y", "8"],
            env=env)
    assert r.returncode == 1
    assert "no CUDA device" in r.stderr and "***DONE***" in r.stderr
    assert not j.exists() or j.read_text() == ""


def test_option_errors_print_done_sentinel():
    r = run(["bench_matmul", "-d", "gpu0", "-T", "float4", "-n", "256"])
    assert r.returncode == 1 and "journal file must be specified" in r.stderr and "***DONE***" in r.stderr
    r = run(["bench_matmul", "-d", "gpu0", "-j", "x", "-T", "float4", "-n", "256", "-e", "-g", "8"])
    assert r.returncode == 1 and "expectation maximization" in r.stderr


def test_retry_reruns_until_done(tmp_path):
    counter = tmp_path / "count"
    counter.write_text("0")
    script = (f'n=$(cat {counter}); n=$((n+1)); echo $n > {counter}; echo attempt $n; '
              f'[ $n -ge 3 ] && echo "***DONE***"; exit 0')
    r = subprocess.run([os.path.join(BIN, "retry"), "bash", "-c", script], capture_output=True, text=True,
                       timeout=60)
    assert r.returncode == 0
    assert counter.read_text().strip() == "3"
    r = subprocess.run([os.path.join(BIN, "retry"), "bash", "-c", "echo never"], capture_output=True,
                       text=True, timeout=60, env=dict(os.environ, RETRY_MAX="2"))
    assert r.returncode == 1 and "gave up" in r.stderr
