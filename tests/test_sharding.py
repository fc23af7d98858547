"""Multi-rank path on CPU: two gloo ranks shard the dumps of a small
configuration, each correlates its own dumps with the CPU oracle, and the
union of their results must equal the single-process result with every dump
computed exactly once. Also checks the max-over-ranks timing reduction."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from oskar_b200.sharding import dump_of_step, dumps_for_rank, max_over_ranks


def test_dumps_partition():
    for world in (1, 2, 3, 8):
        seen = []
        for r in range(world):
            seen += dumps_for_rank(64, world, r)
        assert sorted(seen) == list(range(64))
    assert dump_of_step(3, 4, 1, 64) == 13
    with pytest.raises(ValueError):
        dumps_for_rank(10, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from golden_cases import c1_oracle, load
        from oracle_lib import oracle
        g = load("c1_vis.npz")
        mine = dumps_for_rank(len(g["ha"]), world, rank)
        sub = dict(g)
        sub["ha"] = g["ha"][mine]
        vis = c1_oracle(sub, oracle())
        np.save(os.path.join(out_dir, "r%d.npy" % rank), vis)
        np.save(os.path.join(out_dir, "d%d.npy" % rank), np.array(mine))
        t = max_over_ranks(1.0 + rank)
        np.save(os.path.join(out_dir, "t%d.npy" % rank), np.array([t]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks(tmp_path):
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)),
                       nprocs=world, join=True, start_method="spawn")
    from golden_cases import load
    g = load("c1_vis.npz")
    got = np.zeros_like(g["vis"])
    count = np.zeros(len(g["ha"]), int)
    for r in range(world):
        d = np.load(tmp_path / ("d%d.npy" % r))
        got[d] = np.load(tmp_path / ("r%d.npy" % r))
        count[d] += 1
        assert np.load(tmp_path / ("t%d.npy" % r))[0] == 2.0
    assert np.all(count == 1)
    assert np.max(np.abs(got - g["vis"])) <= 1e-14 * np.max(np.abs(g["vis"]))


def _lib_worker(rank, world, port, out_dir):
    """Each rank builds its own steps' host inputs with the library's
    sharding helper, up to the point where the kernels would be called."""
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oskar_b200 import workloads
        from oskar_b200.sharding import rank_dump_uvw
        cfg = workloads.c3(num_src=64, num_st=40, num_times=10)
        uvw, dumps = rank_dump_uvw(cfg, world, rank, steps=5)
        for i, d in enumerate(dumps):
            assert np.array_equal(uvw[i], cfg.station_uvw(d))
        gathered = [None] * world
        dist.all_gather_object(gathered, dumps)
        np.save(os.path.join(out_dir, "g%d.npy" % rank),
                np.array(gathered))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_library_helpers(tmp_path):
    world = 2
    mp.start_processes(_lib_worker, args=(world, _free_port(), str(tmp_path)),
                       nprocs=world, join=True, start_method="spawn")
    g0 = np.load(tmp_path / "g0.npy")
    assert np.array_equal(g0, np.load(tmp_path / "g1.npy"))
    # five steps of two ranks cover the ten dumps exactly once
    assert sorted(g0.ravel().tolist()) == list(range(10))


def test_bench_spawns_ranks_dry_run():
    """`bench.py --gpus 2` starts its two ranks itself when no launcher
    did; the CPU dry run reports both and their disjoint dumps."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = {k: v for k, v in os.environ.items()
           if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"),
                        "--gpus", "2", "--dry-run", "--steps", "4",
                        "--warmup", "3"], capture_output=True, text=True,
                       env=env, timeout=300)
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["n_gpus"] == 2 and line["dry_run"]
    d0, d1 = line["dumps_per_rank"]
    assert len(d0) == len(d1) == 4 and not set(d0) & set(d1)
