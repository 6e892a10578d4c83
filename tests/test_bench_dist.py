"""bench.py's own multi-process launch on CPU: `--gpus 2` outside torchrun
starts two ranks (gloo here), each takes its shard of the job's channels by
the cost model, and rank 0 reports the world that formed.  The shards are
disjoint and together are the whole channel set (the 40 stations once per
GPU); a single process takes all 40."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _plan(gpus):
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_PORT")}
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", str(gpus), "--backend", "gloo",
                          "--plan-only"], capture_output=True, text=True, timeout=300, env=env, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    return json.loads(out.stdout.strip().splitlines()[-1])


def test_two_ranks_shard_the_channel_set():
    d = _plan(2)
    assert d["n_gpus"] == 2 and d["channels"] == 80
    a, b = (set(s) for s in d["shards"])
    assert not a & b
    assert a | b == set(range(80))
    assert len(a) == len(b) == 40  # equal costs: weak scaling at 40 channels per GPU


def test_one_process_takes_every_channel():
    d = _plan(1)
    assert d["n_gpus"] == 1 and d["shards"] == [list(range(40))]
