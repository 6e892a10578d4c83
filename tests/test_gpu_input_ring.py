"""The batched runner's input ring: blocks in pinned host memory are copied
into ring slots on their own stream as soon as they are submitted (before the
submit waits for a free frame).  With three blocks in flight, blocks of
changing length, a mix that forms tensor-core channel groups, short-arm banks
and WFM stereo chains, and an admission and a retirement mid-stream, every
output is bit-identical to the same blocks given from pageable memory (staged
through the frame's own buffer), and the ring copy shows in the stage times."""
import numpy as np
import pytest

import gpudemod as G
from gpudemod import synth

pytestmark = pytest.mark.gpu

FS = 10_000_000
BLOCK = 262_144
SEED = synth.CONFIG_SEEDS[2] + 9
KEYS = ("pcm", "audio", "rds", "iq", "n_iq", "phase_count", "history_len", "nco_phase", "stereo", "locked",
        "coherence", "pilot_hz", "err_avg", "pll_path")


def _specs():
    _, chans = synth.mixed_scene(device="cpu", block=BLOCK, seed=SEED)
    want = {"NFM": 6, "AM": 5, "USB": 3, "LSB": 3, "CW": 4}
    specs, sid = [], 1
    for kind, n in want.items():
        for _, off in [c for c in chans if c[0] == kind][:n]:
            rate, taps, bw = synth.MODE_TABLE[kind]
            specs.append((sid, off, bw, rate, taps, G.MODE_BY_NAME[kind], G.CH_AUDIO48K))
            sid += 1
    for k, off in enumerate((-3_150_000.0, 2_850_000.0)):
        specs.append((100 + k, off, 250_000.0, 312_500, 256, G.MODE_WFM_STEREO, G.CH_RDS | G.CH_AUDIO48K))
    return specs


def _run(blocks, pinned, depth=3):
    import torch
    r = G.ChannelRunner(FS, BLOCK, max_channels=64, max_taps=1024)
    specs = _specs()
    live = {s[0]: r.admit(*s) for s in specs[:-1]}
    src = [torch.from_numpy(x).pin_memory() for x in blocks] if pinned else blocks
    outs, tickets, h2d = [], [], []

    def collect():
        outs.append({sid: r.result(sl) for sid, sl in live.items()})
        h2d.append(r.stats()["last_h2d_bytes"])

    try:
        for k, x in enumerate(src):
            tickets.append(r.submit(x))
            if k >= depth - 1:
                r.wait(tickets[k - depth + 1])
                collect()
            if k == 3:
                live[specs[-1][0]] = r.admit(*specs[-1])  # a WFM stereo channel joins
            if k == 5:
                r.retire(live.pop(specs[2][0]))
        for k in range(len(src) - depth + 1, len(src)):
            r.wait(tickets[k])
            collect()
        # one more block with stage times: the ring copy is its own stage
        r.set_profiling(True)
        r.process_block(src[0])
        stages = {name for name, _ in r.stage_times()}
        return outs, h2d, stages
    finally:
        r.close()


def test_ring_equals_frame_staging(cuda):
    scene, _ = synth.mixed_scene(device="cuda", block=BLOCK, seed=SEED)
    lengths = [BLOCK, BLOCK - 777, BLOCK, 200_001, BLOCK, BLOCK - 5, BLOCK, BLOCK, 131_072, BLOCK, BLOCK, BLOCK]
    blocks = [scene.next_block().cpu().numpy()[:n] for n in lengths]
    plain, h2d_plain, st_plain = _run(blocks, pinned=False)
    ring, h2d_ring, st_ring = _run(blocks, pinned=True)
    assert len(plain) == len(ring) == len(blocks)
    assert h2d_plain == h2d_ring  # the block and the descriptors, either way
    assert "h2d_ring" in st_ring and "h2d_ring" not in st_plain
    for k, (a, b) in enumerate(zip(plain, ring)):
        assert a.keys() == b.keys(), k
        for sid in a:
            for key in KEYS:
                va, vb = a[sid][key], b[sid][key]
                same = np.array_equal(va, vb) if isinstance(va, np.ndarray) else va == vb
                assert same, (k, sid, key)


def test_sources_interleaved_in_one_stream(cuda):
    """Pinned (input ring), pageable (frame staging) and device-resident
    blocks, and an empty block, alternating in one pipelined stream: the ring
    slots advance only for pinned blocks, and every output equals the
    one-block-at-a-time runner's on the same blocks."""
    import torch
    scene, _ = synth.mixed_scene(device="cuda", block=BLOCK, seed=SEED + 1)
    lengths = [BLOCK, BLOCK - 3, 0, BLOCK, 150_001, BLOCK, BLOCK - 1024, BLOCK, BLOCK]
    raw = [scene.next_block().cpu().numpy()[:n] for n in lengths]
    kinds = ["pin", "page", "pin", "dev", "pin", "pin", "page", "dev", "pin"]
    src = []
    for x, kind in zip(raw, kinds):
        if kind == "pin":
            src.append(torch.from_numpy(x).pin_memory())
        elif kind == "dev":
            src.append(torch.from_numpy(x).to("cuda"))
        else:
            src.append(x)
    specs = _specs()[:-1]

    def runner():
        r = G.ChannelRunner(FS, BLOCK, max_channels=64, max_taps=1024)
        return r, {s[0]: r.admit(*s) for s in specs}

    rs, ls = runner()
    rp, lp = runner()
    try:
        want = []
        for x in raw:
            rs.process_block(x)
            want.append({sid: rs.result(sl) for sid, sl in ls.items()})
        got, tickets = [], []
        for k, x in enumerate(src):
            tickets.append(rp.submit(x))
            if k >= 2:
                rp.wait(tickets[k - 2])
                got.append({sid: rp.result(sl) for sid, sl in lp.items()})
        for k in range(len(src) - 2, len(src)):
            rp.wait(tickets[k])
            got.append({sid: rp.result(sl) for sid, sl in lp.items()})
        assert len(got) == len(want)
        for k, (a, b) in enumerate(zip(want, got)):
            for sid in a:
                for key in KEYS:
                    va, vb = a[sid][key], b[sid][key]
                    same = np.array_equal(va, vb) if isinstance(va, np.ndarray) else va == vb
                    assert same, (k, kinds[k], sid, key)
        assert rp.stats()["blocks"] == len(src)
    finally:
        rs.close()
        rp.close()
