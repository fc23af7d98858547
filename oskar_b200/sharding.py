"""Work sharding across GPUs (one process per GPU).

The (time, channel) problems of a simulation are independent, so N ranks
split the dumps (time samples) among themselves with no data-path
collective: rank r takes dumps r, r + N, r + 2N, ... of the run (weak
scaling when every rank processes the same number of dumps per step). The
only collectives are control-plane ones: a barrier around the timed region
and the maximum of the ranks' times, so the reported time is that of the
slowest rank. This replaces the reference's shared work-unit counter
(oskar/interferometer/src/oskar_interferometer_run_block.c:88-103), which
hands (time, chunk) units to device threads of one process.
"""


import os
import socket
import subprocess
import sys


def dumps_for_rank(num_dumps, world, rank):
    """The dumps rank `rank` of `world` processes, in processing order."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank %d of %d" % (rank, world))
    return list(range(rank, num_dumps, world))


def dump_of_step(step, world, rank, num_dumps):
    """Dump processed by `rank` at its `step`-th step (wraps around)."""
    return (rank + step * world) % num_dumps


def max_over_ranks(value):
    """Maximum of a float over all ranks of the default process group (the
    value itself when no group is initialised)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rank_dump_uvw(cfg, world, rank, steps, first_step=0):
    """Host-side inputs of rank `rank`'s steps: the station (u, v, w) of the
    dump each step processes, [steps][3][num_st] FP64, and those dumps. This
    is everything a rank needs beyond the shared sky and E before its kernel
    calls; no data crosses ranks."""
    import numpy as np
    dumps = [dump_of_step(first_step + i, world, rank, cfg.num_times)
             for i in range(steps)]
    uvw = np.stack([cfg.station_uvw(d) for d in dumps]) if steps else \
        np.zeros((0, 3, cfg.num_st))
    return uvw, dumps


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def spawn_ranks(argv, world, extra_env=None):
    """Starts `world` processes of `argv`, one per GPU as torchrun would:
    RANK = LOCAL_RANK = r, WORLD_SIZE, MASTER_ADDR = 127.0.0.1 and a free
    MASTER_PORT in each one's environment. Rank 0's output goes to this
    process's stdout; the others' stdout is discarded (their errors still
    reach stderr). Waits for all and returns the first non-zero exit code,
    0 if every rank succeeded; if one rank fails, the others are ended so
    that none waits forever on a collective."""
    port = free_port()
    procs = []
    for r in range(world):
        env = dict(os.environ)
        env.update({"RANK": str(r), "LOCAL_RANK": str(r),
                    "WORLD_SIZE": str(world), "LOCAL_WORLD_SIZE": str(world),
                    "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
        if extra_env:
            env.update(extra_env)
        out = None if r == 0 else subprocess.DEVNULL
        procs.append(subprocess.Popen(argv, env=env, stdout=out))
    rc = 0
    pending = list(procs)
    while pending:
        for p in list(pending):
            code = p.poll()
            if code is None:
                continue
            pending.remove(p)
            if code != 0 and rc == 0:
                rc = code
                for q in pending:
                    q.terminate()
        if pending:
            try:
                pending[0].wait(timeout=0.2)
            except subprocess.TimeoutExpired:
                pass
    sys.stdout.flush()
    return rc
