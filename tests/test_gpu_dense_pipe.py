"""Dense polyphase extraction, persistent pipelined kernel: channels of every
staging path (decimation dividing 64 or not, two decimations sharing one
polyphase length, a 16-tap arm, float64 row sums of oversampled FM) across
ragged blocks give the oracle's extraction; a device block at an address that
is not 16-byte aligned takes the one-tile-per-CTA kernel and agrees too."""
import numpy as np
import pytest

import gpudemod as G
from gpudemod import synth
from oracle import oracle as O
from signals import rel_l2

pytestmark = pytest.mark.gpu

FS = 10_000_000
BLOCK = 1 << 18
# (taps, decimation, offset Hz, bandwidth Hz, mode): the same polyphase length
# (8) appears with 32, 20 and 40 phases; mode NFM with out_rate >= 4x bandwidth
# takes float64 row sums; a class staging more than 32 rounds of 512 samples
# stays on the one-tile-per-CTA kernel
CLASSES = [
    (256, 32, 300_000.0, 200_000.0, G.MODE_IQ),
    (160, 20, -1_250_000.0, 150_000.0, G.MODE_IQ),
    (320, 40, 2_100_000.0, 50_000.0, G.MODE_NFM),
    (48, 16, -3_300_000.0, 200_000.0, G.MODE_IQ),
    (250, 25, 900_000.0, 120_000.0, G.MODE_IQ),
    (900, 64, -700_000.0, 40_000.0, G.MODE_IQ),   # 64 x 270 staged samples: one-tile-per-CTA kernel
    (500, 32, 3_500_000.0, 100_000.0, G.MODE_IQ),   # 16-tap arms
    (100, 50, 4_000_000.0, 60_000.0, G.MODE_IQ),
]
LENGTHS = [BLOCK, BLOCK - 777, BLOCK - 3, BLOCK - 1]


def _blocks():
    scene, _ = synth.fm_band_scene(block=BLOCK, n_stations=8, seconds=0.3)
    return [scene.next_block().numpy()[:n] for n in LENGTHS]


def _run(blocks, feed):
    r = G.ChannelRunner(FS, BLOCK, max_channels=len(CLASSES), max_taps=1024)
    try:
        r.set_autotune_table([(T, D, G.FORM_DENSE, 0) for T, D, *_ in CLASSES])
        slots, oracles = [], []
        for k, (T, D, off, bw, mode) in enumerate(CLASSES):
            s = r.admit(k + 1, off, bw, FS // D, T, mode, G.CH_EMIT_IQ)
            assert r.channel_form(s)[0] == G.FORM_DENSE
            slots.append(s)
            oracles.append(O.OracleChannel(FS, off, bw, FS // D, T, O.MODE_NFM, rds=False))
        for b, x in enumerate(blocks):
            r.process_block(feed(x))
            for k, (s, oc) in enumerate(zip(slots, oracles)):
                g, w = r.result(s), oc.process(x)
                assert g["n_iq"] == w["iq"].size, (CLASSES[k], b)
                err = rel_l2(g["iq"], w["iq"])
                assert err <= 1e-5, (CLASSES[k], b, err)
    finally:
        r.close()


def test_dense_classes_match_oracle_host_blocks(cuda):
    _run(_blocks(), lambda x: x)


def test_dense_classes_match_oracle_unaligned_device_blocks(cuda):
    import torch

    def feed(x):
        buf = torch.zeros(x.size + 1, dtype=torch.complex64, device="cuda")
        buf[1:] = torch.from_numpy(x).to("cuda")
        view = buf[1:]
        assert view.data_ptr() % 16 == 8
        return view

    _run(_blocks(), feed)
