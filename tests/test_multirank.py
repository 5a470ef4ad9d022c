"""The multi-rank path of bench.py on CPU: two gloo ranks on 127.0.0.1.

Each rank reconstructs its own instance (no collective on the data path); the
only collective is the max over ranks of the timed region, which the job's
rate divides by.  The reference arm runs on rank 0 alone.
"""

import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime
    import json
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    ms = [120.0, 150.0][rank]  # rank 1 is the slower one
    slowest = bench.max_over_ranks(dist, ms, "cpu")
    dist.barrier()
    total = bench.sum_over_ranks(dist, [4.0, 6.0][rank], "cpu")
    fp = [float((7 * k) % 11 + 1) for k in range(20)]
    owner = bench.shard_by_footprint(fp, world)
    res = {"slowest": slowest, "rate": bench.job_rate(world, 3, slowest), "seed": bench.instance_seed(rank),
           "total": total, "mine": [k for k, o in enumerate(owner) if o == rank]}
    dist.destroy_process_group()
    with open(os.path.join(out_dir, "rank%d.json" % rank), "w") as f:
        json.dump(res, f)


def test_two_gloo_ranks_time_by_the_slowest(tmp_path):
    import json
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    r = [json.load(open(tmp_path / ("rank%d.json" % k))) for k in range(2)]
    assert r[0]["slowest"] == r[1]["slowest"] == 150.0
    # the whole job: 2 ranks x 3 reconstructions x 1000 iterations in 150 ms
    assert r[0]["rate"] == pytest.approx(2 * 3 * 1000 / 0.150)
    assert r[0]["seed"] != r[1]["seed"]  # independent instances
    assert r[0]["total"] == r[1]["total"] == 10.0
    # every instance on exactly one rank, each rank computing the same partition
    assert sorted(r[0]["mine"] + r[1]["mine"]) == list(range(20))


def test_footprint_partition_is_balanced_and_deterministic():
    sys.path.insert(0, ROOT)
    import bench
    fp = [5.0, 3.0, 3.0, 2.0, 2.0, 1.0]
    owner = bench.shard_by_footprint(fp, 2)
    assert owner == bench.shard_by_footprint(fp, 2)
    loads = [sum(f for f, o in zip(fp, owner) if o == r) for r in range(2)]
    assert loads == [8.0, 8.0]
    assert bench.shard_by_footprint(fp, 1) == [0] * len(fp)


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(None, 42.0, "cpu") == 42.0


def test_reference_arm_runs_on_rank_zero_only(capsys):
    sys.path.insert(0, ROOT)
    import bench
    assert bench.run_reference(None, 1, 2) is None  # rank 1 returns at once, prints nothing
    assert capsys.readouterr().out == ""
