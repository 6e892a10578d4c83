"""Dense-form classes too small for the persistent kernel share one launch
(k_extract_dense_any, classes bucketed by shared memory): channels of four
arm lengths in one runner match the oracle, and each channel's IQ is bit for
bit the same as when it runs alone (one class: the per-arm-length kernel)."""
import numpy as np
import pytest

import gpudemod as G
from oracle import oracle as O
from signals import rel_l2

pytestmark = pytest.mark.gpu

FS = 10_000_000
BLOCK = 200_000
# (offset, bandwidth, out rate, taps): D = 40, 50, 80, 64 with L = 5, 6, 10, 13
# (arms of at most four taps take the short-arm form, not the dense one)
CHANS = [(-2_100_000.0, 60_000.0, 250_000, 200), (1_300_000.0, 50_000.0, 200_000, 300),
         (3_700_000.0, 30_000.0, 125_000, 800), (-600_000.0, 25_000.0, 156_250, 832)]


def _blocks():
    """A tone inside every channel's passband plus weak noise, as one
    continuous stream cut into blocks of changing length (stopband-only
    outputs would be rounding noise, not a parity check)."""
    rng = np.random.default_rng(7)
    out, t0 = [], 0
    for b in range(3):
        n = BLOCK - 37 * b
        t = np.arange(t0, t0 + n, dtype=np.float64)
        x = 0.01 * (rng.standard_normal(n) + 1j * rng.standard_normal(n))
        for o, bw, _, _ in CHANS:
            x = x + 0.5 * np.exp(2j * np.pi * (o + 0.2 * bw) * t / FS)
        out.append(x.astype(np.complex64))
        t0 += n
    return out


def _run(chans, blocks):
    r = G.ChannelRunner(FS, BLOCK, max_channels=8, max_taps=2048)
    r.set_channel_groups(False)
    r.set_profiling(True)
    try:
        slots = [r.admit(k + 1, o, bw, rate, t, G.MODE_IQ, G.CH_EMIT_IQ) for k, (o, bw, rate, t) in enumerate(chans)]
        forms = [r.channel_form(s)[0] for s in slots]
        outs, stages = [], set()
        for x in blocks:
            r.process_block(x)
            outs.append([r.result(s)["iq"].copy() for s in slots])
            stages |= {name for name, _ in r.stage_times()}
        return outs, forms, stages
    finally:
        r.close()


def test_dense_classes_in_one_launch(cuda):
    blocks = _blocks()
    mix, forms, stages = _run(CHANS, blocks)
    assert all(f == G.FORM_DENSE for f in forms), forms
    assert "extract_dense" in stages, stages  # the shared launch ran
    refs = [O.OracleChannel(FS, o, bw, rate, t, O.MODE_IQ, rds=False) for o, bw, rate, t in CHANS]
    for b, x in enumerate(blocks):
        for k, ref in enumerate(refs):
            want = ref.process(x)["iq"]
            assert mix[b][k].size == want.size and rel_l2(mix[b][k], want) <= 1e-5, (b, k)
    for k, c in enumerate(CHANS):
        alone, _, st = _run([c], blocks)
        assert "extract_dense" not in st
        for b in range(len(blocks)):
            assert np.array_equal(alone[b][0], mix[b][k]), (k, b)
