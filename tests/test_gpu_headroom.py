"""Channels of the headroom stress mix (61.44 MS/s, FIR lengths 64..1024,
decimation 16..2400, WFM stereo + RDS at D 192) in one batch on the GPU
runner, each against its own oracle chain, block by block.

Some of these channels are ill-conditioned for the FM discriminator: a narrow
filter at a high output rate (NFM, 870 taps, D 30: 12.5 kHz of signal at
2.048 MS/s) leaves consecutive samples nearly equal, and the float32 rounding
of the extraction, magnified by the phase difference, already puts the
reference's own CPU path 1.8e-5 (relative L2) away from the float64 truth of
the same chain.  No float32 implementation with another rounding order can
then be within 1e-5 of it.  For such outputs (the reference's error against
the float64 truth above 5e-6) the bar is accuracy: the GPU output is no
further from the float64 truth than the reference's own."""
import numpy as np
import pytest

import gpudemod as G
from gpudemod import serving as SV
from gpudemod import synth
from oracle import oracle as O
from oracle.truth64 import Truth64Channel
from signals import rel_l2

pytestmark = pytest.mark.gpu

OMODE = {"WFM": O.MODE_WFM_STEREO, "NFM": O.MODE_NFM, "AM": O.MODE_AM, "USB": O.MODE_USB, "LSB": O.MODE_LSB,
         "CW": O.MODE_CW}


def test_headroom_mix_matches_oracle(cuda):
    fs, block = synth.HEADROOM_FS, 1 << 18
    scene, wfm_offs, narrow = synth.headroom_scene(device="cuda", block=block, seconds=0.2)
    mix = SV.HeadroomMix(11, wfm_offs, narrow)
    reqs = [mix.draw() for _ in range(40)]
    # the extremes of the ranges as well: longest filter at the smallest ratio
    # (64 taps per arm), shortest at the largest (one arm)
    reqs.append(SV.Request(1001, 0, 1e9, 1.1e6, "NFM", out_rate=fs // 16, taps=1024, pcm=False))
    reqs.append(SV.Request(1002, 0, 1e9, -2.3e6, "AM", out_rate=fs // 2400, taps=64, pcm=False))
    r = G.ChannelRunner(fs, block, max_channels=64, max_taps=1024)
    slots, oracles, truths = [], [], []
    for q in reqs:
        spec = SV.channel_spec(q)
        slots.append(r.admit(*spec[:6], spec[6] | G.CH_EMIT_IQ))
        args = (fs, q.offset_hz, spec[2], q.out_rate, q.taps, OMODE[q.kind])
        oracles.append(O.OracleChannel(*args, rds=q.kind == "WFM"))
        truths.append(Truth64Channel(*args, rds=q.kind == "WFM"))
    conditioned = 0
    try:
        for b in range(2):
            x = scene.next_block().cpu().numpy()[: block - 1237 * b]
            r.process_block(x)
            for q, sl, oc, tc in zip(reqs, slots, oracles, truths):
                g, w, t = r.result(sl), oc.process(x), tc.process(x)
                ctx = (b, q.kind, q.taps, fs // q.out_rate)
                assert g["n_iq"] == w["iq"].size, ctx
                assert g["audio"].size == w["audio"].size, ctx
                assert g["rds"].size == w["rds"].size, ctx
                for key in ("iq", "audio", "rds"):
                    if not w[key].size:
                        continue
                    e_ref = rel_l2(g[key], w[key])
                    if e_ref <= 1e-5:
                        continue
                    e_truth, e_own = rel_l2(g[key], t[key]), rel_l2(w[key], t[key])
                    assert e_own > 5e-6 and e_truth <= e_own, (ctx, key, e_ref, e_truth, e_own)
                    conditioned += 1
    finally:
        r.close()
    assert conditioned <= 8  # a handful of outputs, not the rule
