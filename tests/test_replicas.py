"""bench.py's multi-GPU path is replicas only: no collective touches the data, ranks only agree on
the slowest time. Run with two gloo ranks on the CPU (the NCCL run uses the same function)."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT

sys.path.insert(0, ROOT)


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = 100.0 + 50.0 * rank          # rank 1 is the slowest
    res = bench.replica_summary(dist, mine, 10.0 * (rank + 1), steps=10, block=1000, world=world)
    with open(os.path.join(out_dir, "r%d.json" % rank), "w") as f:
        json.dump(res, f)
    dist.destroy_process_group()


def test_replica_summary_takes_the_slowest_rank(tmp_path):
    import torch.multiprocessing as mp
    port = 29500 + os.getpid() % 1000
    mp.spawn(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    for r in range(2):
        total, e2e, value = json.load(open(tmp_path / ("r%d.json" % r)))
        assert total == 150.0 and e2e == 20.0
        assert value == pytest.approx(150.0 / (2 * 10 * 1000))


def test_reference_arm_other_ranks_exit_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_single_rank_summary_without_process_group():
    import bench
    assert bench.replica_summary(None, 80.0, 9.0, steps=4, block=500, world=1) == (80.0, 9.0, 80.0 / 2000)


def test_default_line_runs_every_other_configuration(monkeypatch):
    """The default (8M, one GPU) line carries a short run of each other configuration, each through
    its own workload's code path with at least 3 warm-up steps."""
    import argparse
    import bench
    calls = []

    def fake(args, rank, world, local):
        calls.append((args.workload, args.steps, args.warmup))
        return {"workload": args.workload}

    monkeypatch.setattr(bench, "run_prp_config", fake)
    monkeypatch.setattr(bench, "run_batch64", fake)
    args = argparse.Namespace(workload="prp8m", steps=10, warmup=3, block=1000, no_cpu_baseline=False)
    out = bench.other_configs(args, 0, 1, 0)
    assert sorted(out) == ["batch64", "prp20m", "prp256k"]
    assert all(out[w]["workload"] == w for w in out)
    assert all(s >= 1 and w >= 3 for _, s, w in calls)
    assert args.workload == "prp8m" and args.steps == 10      # the caller's arguments are left alone
