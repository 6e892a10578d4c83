"""Dense polyphase extraction, persistent pipelined kernel: classes of every
staging path (decimation dividing 64 or not, two decimations sharing one
polyphase length, 16-tap arms, float64 row sums of oversampled FM), each
large enough for the persistent kernel (two tiles per SM), across ragged
blocks give the oracle's extraction; a device block at an address that is not
16-byte aligned takes the one-tile-per-CTA kernel and agrees too.  No class
has four channels of one decimation divisible by 4, so none is grouped onto
the tensor cores."""
import numpy as np
import pytest

import gpudemod as G
from gpudemod import synth
from oracle import oracle as O
from signals import rel_l2

pytestmark = pytest.mark.gpu

FS = 10_000_000
BLOCK = 1 << 20
# (taps, decimation, bandwidth Hz, mode, channels): the same polyphase length
# (8) appears with 32, 20 and 40 phases; mode NFM with out_rate >= 4x bandwidth
# takes float64 row sums; a class staging more than 64 rounds of 256 samples
# (64 phases x 270) stays on the one-tile-per-CTA kernel
CLASSES = [
    (256, 32, 200_000.0, G.MODE_IQ, 3),
    (160, 20, 150_000.0, G.MODE_IQ, 3),
    (320, 40, 50_000.0, G.MODE_NFM, 3),
    (48, 16, 200_000.0, G.MODE_IQ, 3),
    (250, 25, 120_000.0, G.MODE_IQ, 3),
    (900, 64, 40_000.0, G.MODE_IQ, 1),
    (500, 32, 100_000.0, G.MODE_IQ, 3),
    (100, 50, 60_000.0, G.MODE_IQ, 4),
]
LENGTHS = [BLOCK, BLOCK - 777, BLOCK - 3, BLOCK - 1]


def _blocks():
    scene, _ = synth.fm_band_scene(block=BLOCK, n_stations=8, seconds=0.5)
    return [scene.next_block().numpy()[:n] for n in LENGTHS]


def _run(blocks, feed):
    rng = np.random.default_rng(5)
    chans = [(T, D, bw, mode, float(rng.uniform(-4.5e6, 4.5e6)))
             for T, D, bw, mode, k in CLASSES for _ in range(k)]
    r = G.ChannelRunner(FS, BLOCK, max_channels=len(chans), max_taps=1024)
    try:
        r.set_autotune_table([(T, D, G.FORM_DENSE, 0) for T, D, *_ in CLASSES])
        slots, oracles = [], []
        for k, (T, D, bw, mode, off) in enumerate(chans):
            s = r.admit(k + 1, off, bw, FS // D, T, mode, G.CH_EMIT_IQ)
            assert r.channel_form(s)[0] == G.FORM_DENSE
            slots.append(s)
            oracles.append(O.OracleChannel(FS, off, bw, FS // D, T, O.MODE_NFM, rds=False))
        for b, x in enumerate(blocks):
            r.process_block(feed(x))
            for k, (s, oc) in enumerate(zip(slots, oracles)):
                g, w = r.result(s), oc.process(x)
                assert g["n_iq"] == w["iq"].size, (chans[k], b)
                err = rel_l2(g["iq"], w["iq"])
                assert err <= 1e-5, (chans[k], b, err)
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
