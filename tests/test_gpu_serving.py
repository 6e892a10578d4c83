"""Serving under churn on the GPU: channels joining and leaving at block
boundaries leave every other channel's output unchanged -- each result is the
same alone and in the mix."""
import numpy as np
import pytest

import gpudemod as G
from gpudemod import serving as SV
from gpudemod import synth

pytestmark = pytest.mark.gpu

FS, BLOCK = 10_000_000, 262_144


def _blocks(n):
    scene, stations = synth.serving_scene(device="cuda", block=BLOCK, seconds=n * BLOCK / FS + 1)
    return [scene.next_block().cpu().numpy() for _ in range(n)], stations


def test_results_identical_alone_and_in_churning_mix(cuda):
    blocks, stations = _blocks(6)
    period = BLOCK / FS
    wfm = [st for st in stations if isinstance(st, synth.WFMStation)]
    narrow = [st for st in stations if isinstance(st, synth.NarrowStation)]
    # long-lived channels on stations, plus churn at random frequencies
    reqs = [SV.Request(1, 0.0, 1e9, wfm[0].offset_hz, "WFM"),
            SV.Request(2, 0.0, 1e9, narrow[0].offset_hz, narrow[0].kind),
            SV.Request(3, 1.5 * period, 1e9, wfm[1].offset_hz, "WFM"),         # joins at block 2
            SV.Request(4, 0.0, 2.5 * period, 1_234_567.0, "NFM"),              # leaves after block 2
            SV.Request(5, 0.5 * period, 3.5 * period, -2_345_678.0, "WFM"),    # noise only, joins and leaves
            SV.Request(6, 2.5 * period, 1e9, -777_777.0, "CW"),
            SV.Request(7, 3.5 * period, 1e9, narrow[1].offset_hz, narrow[1].kind)]
    mix = G.ChannelRunner(FS, BLOCK, max_channels=16, max_taps=1024)
    loop = SV.ServingLoop(mix, BLOCK, FS)
    got = {}
    try:
        for k, x in enumerate(blocks):
            t = k * period
            loop.boundary(t, [q for q in reqs if (k - 1) * period < q.t_arrive <= t] if k else
                          [q for q in reqs if q.t_arrive <= 0.0])
            loop.process(x)
            for rid, (slot, _) in loop.live.items():
                got.setdefault(rid, {})[k] = mix.result(slot)
        assert loop.admitted == 7 and loop.retired == 2
        for q in reqs:
            alone = G.ChannelRunner(FS, BLOCK, max_channels=2, max_taps=1024)
            slot = alone.admit(*SV.channel_spec(q))
            try:
                # alone, the channel sees the same blocks from the one it joined at
                for k in sorted(got[q.rid]):
                    alone.process_block(blocks[k])
                    a, m = alone.result(slot), got[q.rid][k]
                    assert m["pcm"].size > 0 or m["n_iq"] == 0
                    for key in ("pcm", "audio", "rds"):
                        assert np.array_equal(a[key], m[key]), (q.rid, k, key)
                    assert a["stereo"] == m["stereo"] and a["locked"] == m["locked"], (q.rid, k)
            finally:
                alone.close()
    finally:
        mix.close()
