"""Host logic of bench.py's multi-rank path on CPU (gloo, world size 2).

On a GPU node bench.py runs one replica per rank (NCCL); what does not need a
GPU is checked here: the max-over-ranks reduction of the timings, the barrier,
and the reference arm, which only rank 0 runs and prints.
"""

import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_MAX_OVER_RANKS = r"""
import os, sys, json, argparse, torch
sys.path.insert(0, {root!r})
import bench
args = argparse.Namespace(impl="reference")
world, rank, local = bench.dist_init(args)
bench.barrier(world)
m = bench.max_over_ranks(10.0 + 5.0 * rank, world, torch.device("cpu"))
bench.barrier(world)
import torch.distributed as dist
dist.destroy_process_group()
print(json.dumps({{"rank": rank, "world": world, "max": m}}))
"""

_REFERENCE_ARM = r"""
import os, sys, argparse
sys.path.insert(0, {root!r})
import bench
# a tiny kooshball so the oracle finishes in seconds
bench.WORKLOAD = dict(N=16, coils=2, spokes=40, samples=32, width=4, oversamp=1.25)
args = argparse.Namespace(impl="reference", steps=1, warmup=0, small=False, medium=False)
bench.run_reference(args)
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _launch(code, world):
    port = _free_port()
    procs = []
    for rank in range(world):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                   LOCAL_RANK=str(rank), WORLD_SIZE=str(world), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", code.format(root=ROOT)], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=240)
        assert p.returncode == 0, err[-2000:]
        outs.append(out)
    return outs


@pytest.mark.timeout(300)
def test_max_over_ranks_two_gloo_ranks():
    outs = _launch(_MAX_OVER_RANKS, 2)
    res = [json.loads(o.strip().splitlines()[-1]) for o in outs]
    assert sorted(r["rank"] for r in res) == [0, 1]
    assert all(r["world"] == 2 and r["max"] == 15.0 for r in res)


@pytest.mark.timeout(300)
def test_reference_arm_only_rank0_prints():
    outs = _launch(_REFERENCE_ARM, 2)
    line = json.loads(outs[0].strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"
    assert outs[1].strip() == ""
