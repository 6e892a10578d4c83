"""Tensor-core extraction of channel groups (gemm_extract.cu): channels that
share decimation, tap count and phase count are extracted as one TF32x3 GEMM
on tcgen05; groups of several sizes (padded columns, a partial last tile) and
the channels left on the dense kernel (too few to group, decimation not a
multiple of 4) all give the oracle's extraction across ragged blocks, and the
group kernel is the one that ran."""
import numpy as np
import pytest

import gpudemod as G
from gpudemod import synth
from oracle import oracle as O
from signals import rel_l2

pytestmark = pytest.mark.gpu

FS = 10_000_000
BLOCK = 1 << 18
LENGTHS = [BLOCK, BLOCK - 777, BLOCK - 3, BLOCK - 32]


def _specs():
    rng = np.random.default_rng(11)
    out = []
    # 12 channels of (256 taps, D 32): one group, N = 32
    for _ in range(12):
        out.append((256, 32, float(rng.uniform(-4.5e6, 4.5e6)), float(rng.uniform(80e3, 250e3))))
    # 5 channels of (100 taps, D 20): one group of 5, N = 16 (6 padded columns)
    for _ in range(5):
        out.append((100, 20, float(rng.uniform(-4.5e6, 4.5e6)), float(rng.uniform(40e3, 150e3))))
    # 3 channels of (64, 16): too few, dense kernel
    for _ in range(3):
        out.append((64, 16, float(rng.uniform(-4.5e6, 4.5e6)), 100e3))
    # 4 channels of (250, 25): decimation not a multiple of 4, dense kernel
    for _ in range(4):
        out.append((250, 25, float(rng.uniform(-4.5e6, 4.5e6)), 120e3))
    return out


def test_groups_match_oracle(cuda):
    scene, _ = synth.fm_band_scene(block=BLOCK, n_stations=8, seconds=0.3)
    blocks = [scene.next_block().numpy()[:n] for n in LENGTHS]
    specs = _specs()
    r = G.ChannelRunner(FS, BLOCK, max_channels=len(specs), max_taps=1024)
    try:
        r.set_autotune_table([(T, D, G.FORM_DENSE, 0) for T, D in {(s[0], s[1]) for s in specs}])
        r.set_profiling(True)
        slots, oracles = [], []
        for k, (T, D, off, bw) in enumerate(specs):
            s = r.admit(k + 1, off, bw, FS // D, T, G.MODE_IQ, G.CH_EMIT_IQ)
            assert r.channel_form(s)[0] == G.FORM_DENSE
            slots.append(s)
            oracles.append(O.OracleChannel(FS, off, bw, FS // D, T, O.MODE_NFM, rds=False))
        for b, x in enumerate(blocks):
            r.process_block(x)
            names = [n for n, _ in r.stage_times()]
            assert "extract_gemm" in names, names
            for k, (s, oc) in enumerate(zip(slots, oracles)):
                g, w = r.result(s), oc.process(x)
                assert g["n_iq"] == w["iq"].size, (specs[k], b)
                err = rel_l2(g["iq"], w["iq"])
                assert err <= 1e-5, (specs[k], b, err)
    finally:
        r.close()


def test_groups_switch_and_mix_invariance(cuda):
    """With channel groups off a channel's IQ is bit-identical alone and in a
    mix that would form a group; with them on the grouped IQ stays within the
    parity bar of the ungrouped one."""
    scene, _ = synth.fm_band_scene(block=BLOCK, n_stations=8, seconds=0.3)
    blocks = [scene.next_block().numpy()[:n] for n in LENGTHS[:3]]
    rng = np.random.default_rng(3)
    specs = [(k + 1, float(rng.uniform(-4.5e6, 4.5e6)), 200e3, FS // 32, 256, G.MODE_IQ, G.CH_EMIT_IQ)
             for k in range(6)]

    def run(channels, groups):
        r = G.ChannelRunner(FS, BLOCK, max_channels=8, max_taps=1024)
        try:
            r.set_channel_groups(groups)
            r.set_profiling(True)
            slots = [r.admit(*s) for s in channels]
            out, grouped = [], False
            for x in blocks:
                r.process_block(x)
                grouped |= "extract_gemm" in [n for n, _ in r.stage_times()]
                out.append(r.result(slots[0])["iq"].copy())
            return out, grouped
        finally:
            r.close()

    alone, g0 = run(specs[:1], True)
    assert not g0
    off, g1 = run(specs, False)
    assert not g1
    on, g2 = run(specs, True)
    assert g2
    for a, b, c in zip(alone, off, on):
        assert np.array_equal(a, b)
        assert rel_l2(c, a) <= 1e-5



def test_group_taps_follow_retune(cuda):
    """The packed group taps are cached per frame (three frames): retunes of
    members between blocks -- offset only, bandwidth only (new taps), both --
    reach the group kernel on the next block in every frame; the grouped
    runner stays within the parity bar of one with groups off that gets the
    same calls."""
    scene, _ = synth.fm_band_scene(block=BLOCK, n_stations=8, seconds=0.8)
    blocks = [scene.next_block().numpy() for _ in range(9)]
    rng = np.random.default_rng(9)
    offs = [float(rng.uniform(-4.5e6, 4.5e6)) for _ in range(6)]
    calls = {2: [(1, offs[1] + 777.0, 200e3)], 4: [(2, offs[2], 120e3)], 5: [(3, offs[3] - 2500.0, 90e3)]}

    def run(groups):
        r = G.ChannelRunner(FS, BLOCK, max_channels=8, max_taps=1024)
        try:
            r.set_channel_groups(groups)
            r.set_profiling(True)
            slots = [r.admit(k + 1, off, 200e3, FS // 32, 256, G.MODE_IQ, G.CH_EMIT_IQ)
                     for k, off in enumerate(offs)]
            out = []
            for b, x in enumerate(blocks):
                for k, off, bw in calls.get(b, []):
                    r.update(slots[k], off, bw)
                r.process_block(x)
                assert ("extract_gemm" in [n for n, _ in r.stage_times()]) == groups
                out.append([r.result(s)["iq"].copy() for s in slots])
            return out
        finally:
            r.close()

    on, off = run(True), run(False)
    for b, (a, c) in enumerate(zip(on, off)):
        for k, (x, y) in enumerate(zip(a, c)):
            assert rel_l2(x, y) <= 1e-5, (b, k, rel_l2(x, y))


def test_fm_band_group_matches_oracle(cuda):
    """The FM band geometry: 40 WFM stereo stations of 256 taps at decimation
    32 from 10 MS/s in 2^20-sample blocks form one 80-column group whose tiles
    stage their block span by bulk copy; every channel's IQ and, for four of
    them, the stereo audio and RDS baseband match the oracle."""
    block = 1 << 20
    scene, st = synth.fm_band_scene(block=block, n_stations=40, seconds=0.3)
    r = G.ChannelRunner(FS, block, max_channels=40, max_taps=1024)
    try:
        r.set_profiling(True)
        slots = [r.admit(k + 1, s.offset_hz, 250_000.0, 312_500, 256, G.MODE_WFM_STEREO, G.CH_RDS | G.CH_EMIT_IQ)
                 for k, s in enumerate(st)]
        iq_or = [O.OracleChannel(FS, s.offset_hz, 250_000.0, 312_500, 256, O.MODE_NFM, rds=False) for s in st]
        full = {k: O.OracleChannel(FS, st[k].offset_hz, 250_000.0, 312_500, 256, O.MODE_WFM_STEREO, rds=True)
                for k in (0, 13, 26, 39)}
        for b in range(2):
            x = scene.next_block().numpy()
            r.process_block(x)
            assert "extract_gemm" in [n for n, _ in r.stage_times()]
            for k, (s, oc) in enumerate(zip(slots, iq_or)):
                g, w = r.result(s), oc.process(x)
                assert g["n_iq"] == w["iq"].size
                assert rel_l2(g["iq"], w["iq"]) <= 1e-5, (k, b, rel_l2(g["iq"], w["iq"]))
                if k in full:
                    wf = full[k].process(x)
                    assert rel_l2(g["audio"], wf["audio"]) <= 1e-5, (k, b, rel_l2(g["audio"], wf["audio"]))
                    assert rel_l2(g["rds"], wf["rds"]) <= 1e-5, (k, b, rel_l2(g["rds"], wf["rds"]))
    finally:
        r.close()
