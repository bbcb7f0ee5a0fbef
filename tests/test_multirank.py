"""The N > 1 path of bench.py on CPU: two ranks over gloo (one process each, rendezvous on
127.0.0.1), running the bench's own rank plumbing.

* Each rank solves its own right-hand sides: the seeds of the ranks are disjoint and together
  2 .. 1 + 32·N, rank r holding 2 + 32r .. 1 + 32(r + 1).
* The timing is the max over ranks and the whole-job rate counts every rank's solves over it.
* The reference arm runs on rank 0 only: the other ranks return at once and print nothing.
* Every rank takes the same collective steps (barrier, max-reduction) and leaves the group.
"""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import argparse, io, json, sys, contextlib, time
sys.path.insert(0, sys.argv[1])
import bench
import torch.distributed as dist

world, rank, local = bench.dist_env()
bench.init_dist(world, "gloo", timeout_s=60)
barrier, max_over_ranks = bench.collectives(world, "cpu")
seeds = bench.rank_seeds(rank)
every = [None] * world
dist.all_gather_object(every, seeds)
barrier()
slowest = max_over_ranks(1.0 + rank)
rate = bench.whole_job_rate(bench.NRHS, world, 10, slowest)
out = io.StringIO()
t0 = time.perf_counter()
with contextlib.redirect_stdout(out):
    ref = bench.run_reference(argparse.Namespace(steps=1, warmup=0)) if rank != 0 else None
ref_seconds = time.perf_counter() - t0
barrier()
dist.destroy_process_group()
print(json.dumps({"rank": rank, "seeds": every, "slowest": slowest, "rate": rate,
                  "ref_output": out.getvalue(), "ref_seconds": ref_seconds}))
"""


def _free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.timeout(240)
def test_two_gloo_ranks_run_the_bench_plumbing():
    world = 2
    port = _free_port()
    procs = []
    for rank in range(world):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", WORKER, ROOT], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    results = []
    try:
        for p in procs:
            out, err = p.communicate(timeout=200)
            assert p.returncode == 0, err[-2000:]
            results.append(json.loads(out.strip().splitlines()[-1]))
    finally:
        for p in procs:
            if p.poll() is None:
                p.kill()
    results.sort(key=lambda r: r["rank"])
    n = 32
    for r in results:
        assert r["seeds"][0] == list(range(2, 2 + n)) and r["seeds"][1] == list(range(2 + n, 2 + 2 * n))
        assert r["slowest"] == 2.0                     # max over ranks of 1.0 + rank
        assert r["rate"] == n * world * 10 / 2.0       # every rank's solves over the slowest time
    assert results[1]["ref_output"] == "" and results[1]["ref_seconds"] < 5.0
