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
