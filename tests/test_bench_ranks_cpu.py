"""The multi-rank plumbing of bench.py on CPU (gloo, world size 2): the timing
of the job is the maximum over the ranks' timings, and under torchrun the
reference arm runs on rank 0 alone while the other ranks leave without work
or output.  The path does not shard (one independent replica per GPU), so
these are the only cross-rank steps."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


_WORKER = r"""
import os, sys, json, datetime
sys.path.insert(0, {root!r})
import torch.distributed as dist
import bench
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
rank, world, _ = bench.dist_env()
got = bench.max_over_ranks([1.0 + rank, 10.0 - rank, 5.0], world, device="cpu")
dist.barrier()
dist.destroy_process_group()
print(json.dumps({{"rank": rank, "got": got}}))
"""


def test_timings_are_the_maximum_over_ranks():
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", _WORKER.format(root=ROOT)], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            out, err = p.communicate(timeout=180)
        except subprocess.TimeoutExpired:
            p.kill()
            raise
        assert p.returncode == 0, err[-2000:]
        outs.append(out)
    import json

    for out in outs:
        line = json.loads(out.strip().splitlines()[-1])
        assert line["got"] == [2.0, 10.0, 5.0]


def test_single_rank_needs_no_collective():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks([3, 4.5], 1) == [3.0, 4.5]


@pytest.mark.parametrize("rank", [1])
def test_reference_arm_runs_on_rank_zero_only(rank):
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank), CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""
