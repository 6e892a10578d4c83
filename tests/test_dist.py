"""Multi-process path (world size 2, gloo on CPU): channel sharding across
ranks, no data-path collective, barrier + max-reduced timing.  Each rank runs
its shard through the oracle chain; the union equals the single-process run
(sharding never changes a channel's output)."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from gpudemod import dist as D

FS, BLOCK = 2_400_000, 65_536
SPECS = [(300_000.0, 250_000.0, 300_000, 128, 3), (-450_000.0, 12_500.0, 25_000, 512, 1),
         (700_000.0, 10_000.0, 25_000, 384, 4), (-900_000.0, 3_000.0, 12_500, 256, 5),
         (100_000.0, 500.0, 5_000, 128, 7)]


def _blocks():
    from gpudemod import synth
    scene, _ = synth.plain_wfm_scene(block=BLOCK)
    return [scene.next_block().numpy() for _ in range(2)]


def _run(specs_idx, blocks):
    from oracle import oracle as O
    out = {}
    for i in specs_idx:
        off, bw, rate, taps, mode = SPECS[i]
        ch = O.OracleChannel(FS, off, bw, rate, taps, mode, rds=(mode == 3))
        out[i] = [ch.process(b)["audio"] for b in blocks]
    return out


def _worker(rank, world, port, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "argus-sdr_b200")):
        if p not in sys.path:
            sys.path.insert(0, p)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    from gpudemod import dist as DD
    w, r, _ = DD.init("gloo", timeout_s=60)
    costs = [DD.channel_cost(BLOCK, FS // s[2], s[3], s[4]) for s in SPECS]
    shard = DD.partition_channels(costs, w)[r]
    blocks = _blocks()
    DD.barrier(w)
    res = _run(shard, blocks)
    t = DD.max_over_ranks(w, float(r + 1))
    DD.barrier(w)
    q.put((r, shard, t, {k: [a.tolist() for a in v] for k, v in res.items()}))
    import torch.distributed as dist
    dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_partition_balances_and_covers():
    costs = [D.channel_cost(BLOCK, FS // s[2], s[3], s[4]) for s in SPECS]
    shards = D.partition_channels(costs, 2)
    assert sorted(i for s in shards for i in s) == list(range(len(SPECS)))
    loads = [sum(costs[i] for i in s) for s in shards]
    assert max(loads) <= sum(loads) / 2 + max(costs)  # list-scheduling bound


def test_two_rank_sharded_run_matches_single_process():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    shards = {r: sh for r, sh, _, _ in got}
    assert sorted(shards[0] + shards[1]) == list(range(len(SPECS)))
    assert all(t == 2.0 for _, _, t, _ in got)  # max over ranks
    single = _run(range(len(SPECS)), _blocks())
    for _, _, _, res in got:
        for k, v in res.items():
            for a, b in zip(v, single[int(k)]):
                assert np.array_equal(np.asarray(a, np.float32), b)
