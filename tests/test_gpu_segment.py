"""One-shot segment demod on the GPU (gpud_demod_audio_segment) against the
oracle's restatement of demodAudioCPU (recorder/cpu_audio.go:10-75) -- the
live /api/demod path and event recordings: shift, 101-tap low-pass,
decimation to ~48 kHz (~192 kHz for WFM), the mode's demodulator (WFM_STEREO:
demod.wfmStereo's free-running 38 kHz carrier, demod/fm.go:92-123), then the
63-tap anti-alias stage above 48 kHz."""
import numpy as np
import pytest

import gpudemod as G
from gpudemod import synth
from oracle import oracle as O
from signals import rel_l2

pytestmark = pytest.mark.gpu

MODES = {"NFM": (G.MODE_NFM, O.MODE_NFM), "AM": (G.MODE_AM, O.MODE_AM), "USB": (G.MODE_USB, O.MODE_USB),
         "LSB": (G.MODE_LSB, O.MODE_LSB), "CW": (G.MODE_CW, O.MODE_CW), "WFM": (G.MODE_WFM, O.MODE_WFM),
         "WFM_STEREO": (G.MODE_WFM_STEREO, O.MODE_WFM_STEREO)}


def _check(kind, x, fs, off, bw):
    gm, om = MODES[kind]
    a, ch, rate, drate = G.demod_audio_segment(gm, x, fs, off, bw)
    w, wch, wrate, wdrate = O.demod_audio_segment(om, x, fs, off, bw)
    assert (ch, rate, drate) == (wch, wrate, wdrate), kind
    assert a.size == w.size, (kind, a.size, w.size)
    for c in range(ch):
        assert rel_l2(a[c::ch], w[c::ch]) <= 1e-5, (kind, c, rel_l2(a[c::ch], w[c::ch]))
    return a, ch, rate


@pytest.mark.parametrize("kind", ["NFM", "AM", "USB", "LSB", "CW"])
def test_narrow_segment_10msps(cuda, kind):
    scene, chans = synth.mixed_scene(block=1 << 19)
    x = scene.next_block().numpy()
    off = next(o for k, o in chans if k == kind)
    # 10 MS/s: decimation 208 to 48076 S/s, anti-alias stage with d2 = 1
    _, _, rate = _check(kind, x, 10_000_000, off, synth.MODE_TABLE[kind][2])
    assert rate == 10_000_000 // 208


@pytest.mark.parametrize("kind", ["WFM", "WFM_STEREO"])
def test_wideband_segment(cuda, kind):
    scene, _ = synth.plain_wfm_scene(block=262_144)
    x = np.concatenate([scene.next_block().numpy() for _ in range(2)])
    # 2.4 MS/s: 184615 S/s, anti-alias and every 4th frame -> 46153 S/s
    a, ch, rate = _check(kind, x, 2_400_000, 300_000.0, 200_000.0)
    assert rate == 184_615 // 4 and ch == (2 if kind == "WFM_STEREO" else 1)
    if kind == "WFM_STEREO":
        assert not np.allclose(a[0::2], a[1::2])
    # 1.92 MS/s at DC: D 10 to 192000, then 48000 exactly
    _check(kind, x[:300_000], 1_920_000, 0.0, 180_000.0)


def test_segment_without_second_stage(cuda):
    scene, chans = synth.mixed_scene(block=1 << 18)
    x = scene.next_block().numpy()
    off = next(o for k, o in chans if k == "NFM")
    # 1.92 MS/s: D 40 to exactly 48 kHz, no anti-alias stage
    _, _, rate = _check("NFM", x, 1_920_000, off / 5.0, 12_500.0)
    assert rate == 48_000
