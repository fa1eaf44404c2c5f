"""The multi-rank host logic of bench.py on CPU: world size 2 over gloo.

`bench.py --gpus N` runs N independent replicas, one per rank. The timed
region's duration is the maximum over ranks, and a failure on one rank
reaches every rank through the same collective, so no rank waits for one
that gave up. The reference arm runs on rank 0 alone.
"""
import datetime
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, port, values, fails, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE="2",
                      LOCAL_RANK=str(rank))
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=2, timeout=datetime.timedelta(seconds=30))
    try:
        for v, f in zip(values[rank], fails[rank]):
            out.put((rank, bench.max_over_ranks(v, dist, failed=f)))
    finally:
        dist.destroy_process_group()


def _run(values, fails):
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, port, values, fails, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = {}
    while not out.empty():
        r, res = out.get()
        got.setdefault(r, []).append(res)
    return got


def test_max_over_ranks_and_failure_flag_on_two_gloo_ranks():
    got = _run(values={0: [10.0, 3.0], 1: [12.5, 2.0]}, fails={0: [False, False], 1: [False, True]})
    for r in (0, 1):
        assert got[r][0] == (12.5, False)
        assert got[r][1] == (3.0, True)


def test_max_over_ranks_without_a_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(4.0, None) == (4.0, False)
    assert bench.max_over_ranks(4.0, None, failed=True) == (4.0, True)


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""


def test_reference_arm_uses_every_host_core():
    import json
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    if "unavailable" in line:
        return  # neither the compiled reference nor the restatement could run here
    try:
        cores = len(os.sched_getaffinity(0))
    except AttributeError:
        cores = os.cpu_count()
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["cores"] == min(cores, 120)
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]
