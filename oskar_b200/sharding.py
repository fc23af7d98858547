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
