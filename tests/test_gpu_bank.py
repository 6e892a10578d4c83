"""Short-arm channel banks (bank_extract.cu): channels of one decimation, tap
count (at most four taps per arm) and phase count share one staging of the
block.  Every banked channel's IQ against the oracle, block after block
(block lengths that are not multiples of the decimation, so the phase count
moves), with channels that join later (another phase count: another bank),
a class too small for a bank, and the same channels with channel groups
switched off (no banks) within the parity tolerance."""
import numpy as np
import pytest

import gpudemod as G
from gpudemod import synth
from oracle import oracle as O
from signals import rel_l2

pytestmark = pytest.mark.gpu

FS = 10_000_000
TOL = 1e-5
OMODE = {"NFM": O.MODE_NFM, "AM": O.MODE_AM, "USB": O.MODE_USB, "LSB": O.MODE_LSB, "CW": O.MODE_CW}


def _scene_blocks(lengths):
    scene, specs = synth.mixed_scene(device="cuda", block=max(lengths), seed=synth.CONFIG_SEEDS[2] + 5)
    blocks = [scene.next_block().cpu().numpy()[:n] for n in lengths]
    return blocks, specs


def _pick(specs, counts):
    out = []
    for kind, want in counts.items():
        out += [(k, off) for k, off in specs if k == kind][:want]
    return out


def _chan(kind, off):
    out_rate, taps, bw = synth.MODE_TABLE[kind]
    return off, bw, out_rate, taps


@pytest.mark.parametrize("groups_on", [True, False])
def test_banked_channels_match_oracle(cuda, groups_on):
    lengths = [262_144, 250_001, 262_144 - 777, 199_999]
    blocks, specs = _scene_blocks(lengths)
    # NFM / AM / USB+LSB / CW classes of >= 4 channels, and 2 channels of a class too small for a bank
    chans = _pick(specs, {"NFM": 6, "AM": 5, "USB": 3, "LSB": 3, "CW": 4})
    small = [("NFM", -4_400_000.0 + 7_000.0 * i) for i in range(2)]
    late = _pick(specs, {"NFM": 8})[6:8] + _pick(specs, {"AM": 9})[5:9]
    r = G.ChannelRunner(FS, max(lengths), max_channels=64, max_taps=1024)
    r.set_channel_groups(groups_on)
    r.set_profiling(True)
    refs = {}
    try:
        def admit(k, kind, off, taps=None):
            o, bw, rate, t = _chan(kind, off)
            t = taps or t
            slot = r.admit(k, o, bw, rate, t, G.MODE_IQ, G.CH_EMIT_IQ)
            refs[slot] = O.OracleChannel(FS, o, bw, rate, t, OMODE[kind], rds=False)

        for k, (kind, off) in enumerate(chans):
            admit(k + 1, kind, off)
        for k, (kind, off) in enumerate(small):
            admit(100 + k, kind, off, taps=640)  # T = 640, D = 400: its own class of two
        stages = set()
        for b, x in enumerate(blocks):
            if b == 1:
                for k, (kind, off) in enumerate(late):
                    admit(200 + k, kind, off)
            r.process_block(x)
            stages |= {name for name, _ in r.stage_times()}
            for slot, ref in refs.items():
                g, w = r.result(slot)["iq"], ref.process(x)["iq"]
                assert g.size == w.size, (b, slot)
                err = rel_l2(g, w)
                assert err <= TOL, (b, slot, err)
        assert ("extract_bank" in stages) == groups_on
    finally:
        r.close()


def test_bank_equals_unbanked_within_tolerance(cuda):
    """The same channels with and without banks: a banked channel's sums run
    in another order, so their IQ agree within the parity tolerance."""
    lengths = [262_144, 262_144]
    blocks, specs = _scene_blocks(lengths)
    chans = _pick(specs, {"NFM": 5, "CW": 4})
    outs = []
    for on in (True, False):
        r = G.ChannelRunner(FS, max(lengths), max_channels=16, max_taps=1024)
        r.set_channel_groups(on)
        try:
            slots = []
            for k, (kind, off) in enumerate(chans):
                o, bw, rate, t = _chan(kind, off)
                slots.append(r.admit(k + 1, o, bw, rate, t, G.MODE_IQ, G.CH_EMIT_IQ))
            res = []
            for x in blocks:
                r.process_block(x)
                res.append([r.result(s)["iq"].copy() for s in slots])
            outs.append(res)
        finally:
            r.close()
    for blk_on, blk_off in zip(*outs):
        for a, b in zip(blk_on, blk_off):
            assert a.size == b.size and rel_l2(a, b) <= TOL


def test_plain_schedule_with_bankable_channels(cuda):
    """The plain per-signal schedule runs every channel alone, so none is
    banked, while the same set in the batched schedule forms banks; a
    modulated-form class with phase groups (partial sums) among them.  Both
    schedules give every channel's IQ within the parity tolerance."""
    lengths = [262_144, 262_144 - 999]
    blocks, specs = _scene_blocks(lengths)
    chans = _pick(specs, {"NFM": 5, "AM": 5, "CW": 4})
    outs = []
    for sched in (G.SCHED_BATCHED, G.SCHED_PLAIN):
        r = G.ChannelRunner(FS, max(lengths), max_channels=16, max_taps=1024)
        r.set_autotune_table([(384, 400, G.FORM_MOD, 96)])  # AM: modulated form, four phase groups
        r.set_schedule(sched)
        try:
            slots = []
            for k, (kind, off) in enumerate(chans):
                o, bw, rate, t = _chan(kind, off)
                slots.append(r.admit(k + 1, o, bw, rate, t, G.MODE_IQ, G.CH_EMIT_IQ))
            assert r.channel_form(slots[5])[:2] == (G.FORM_MOD, 96)
            res = []
            for x in blocks:
                r.process_block(x)
                res.append([r.result(s)["iq"].copy() for s in slots])
            outs.append(res)
        finally:
            r.close()
    for blk_b, blk_p in zip(*outs):
        for a, b in zip(blk_b, blk_p):
            assert a.size == b.size and rel_l2(a, b) <= TOL
