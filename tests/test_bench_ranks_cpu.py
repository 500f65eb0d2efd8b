"""The multi-GPU host logic of bench.py on CPU: two ranks over gloo (replicas
only, so the one collective is the max-over-ranks of the timings), and the
reference arm under torchrun, where rank 0 alone runs."""
import os
import socket
import subprocess
import sys
import types

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402

CHILD = r"""
import os, sys, datetime
sys.path.insert(0, os.environ["APO_ROOT"])
import torch.distributed as dist
import bench
rank, world, _ = bench.dist_env()
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=30))
mine = [3.5, 7.25][rank]
print("MAX", bench.max_over_ranks(mine, world, "cpu"), flush=True)
print("SEED", bench.replica_seed(rank), flush=True)
dist.barrier()
dist.destroy_process_group()
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_max_over_ranks_with_two_gloo_ranks():
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), APO_ROOT=ROOT)
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=180)
        assert p.returncode == 0, err
        outs.append(out)
    seeds = set()
    for out in outs:
        vals = dict(line.split() for line in out.strip().splitlines())
        assert float(vals["MAX"]) == 7.25          # every rank sees the slowest time
        seeds.add(int(vals["SEED"]))
    assert len(seeds) == 2                          # replicas start from different velocities


def test_single_rank_needs_no_process_group():
    assert bench.max_over_ranks(2.5, 1) == 2.5


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    def no_work(*a, **k):
        raise AssertionError("a rank other than 0 did work")

    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setattr(bench, "make_system", no_work)
    monkeypatch.setattr(bench, "cpu_baseline", no_work)
    args = types.SimpleNamespace(workload="chain23k", gpus=2, steps=1, warmup=3)
    assert bench.run_reference_arm(args) == 0


def test_gpus_flag_relaunches_under_torchrun():
    """`bench.py --gpus 2` outside torchrun starts itself under torchrun with
    two ranks; the reference arm then runs on rank 0 alone (here, without a
    GPU, it times the FP64 host restatement) and prints one line."""
    env = dict(os.environ)
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT"):
        env.pop(k, None)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "3", "--workload", "water12k"],
                       env=env, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    import json
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["config"] == bench.bench_config(bench.WORKLOADS["water12k"], 12480)


def test_gpus_flag_must_match_world_size():
    env = dict(os.environ, RANK="0", WORLD_SIZE="2", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "1"],
                       env=env, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True,
                       timeout=120)
    assert r.returncode == 2
    assert "WORLD_SIZE" in r.stderr
