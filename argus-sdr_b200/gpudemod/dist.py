"""Multi-GPU plumbing for the runner: one process per GPU, channels sharded
across ranks (channels are independent -- no cross-channel reduction exists),
no collective on the data path.  Each rank receives the wideband block itself
(its own H2D); only a barrier and a max-reduction of timings cross ranks.
"""
from __future__ import annotations

import datetime
import os


def env_world():
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: int = 120):
    """Initialise the process group from torchrun's environment.  Returns
    (world, rank, local_rank); world == 1 needs no process group."""
    import torch
    world, rank, local = env_world()
    if world > 1:
        import torch.distributed as dist
        kw = {}
        if backend == "nccl":
            torch.cuda.set_device(local)
            kw["device_id"] = torch.device("cuda", local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    elif backend == "nccl" and torch.cuda.is_available():
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world: int, v: float, device=None) -> float:
    if world <= 1:
        return float(v)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def channel_cost(n_in: int, decim: int, taps: int, mode: int) -> float:
    """Per-block flop estimate of one channel: extraction 4*T*n_out plus the
    rotation of every input sample, plus the demod per composite sample
    (WFM stereo ~1250 flop incl. the 6 stereo filters and the PLL)."""
    n_out = n_in // max(1, decim)
    demod = {0: 0, 1: 6, 2: 208, 3: 1250, 4: 5, 5: 3, 6: 3, 7: 1}.get(mode, 6)
    return 4.0 * taps * n_out + 6.0 * n_in + demod * n_out


def partition_channels(costs, world: int):
    """Longest-processing-time-first assignment of channels to ranks.
    Returns a list (per rank) of channel indices."""
    order = sorted(range(len(costs)), key=lambda i: -costs[i])
    load = [0.0] * world
    shards = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: load[k])
        shards[r].append(i)
        load[r] += costs[i]
    for s in shards:
        s.sort()
    return shards
