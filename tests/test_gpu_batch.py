"""Event-recording batch WFM stereo on the GPU (gpud_wfm_batch_audio) against
the oracle's restatement of demodWFMStereoBatchAudio
(recorder/wfm_batch_stereo.go:10-155): shift, 101-tap low-pass, decimation
round(fs/192000), discriminator, batch stereo decoder (pilot-power-ratio lock,
duplicated mono when not locked), 48 kHz stereo resampler, de-emphasis,
x0.35 -- one stateless call over a whole capture."""
import numpy as np
import pytest

import gpudemod as G
from gpudemod import synth
from oracle import oracle as O
from signals import rel_l2

pytestmark = pytest.mark.gpu


def _check(x, fs, off, bw, tau, want_locked=None):
    a, rate, lk, drate = G.wfm_batch_audio(x, fs, off, bw, tau)
    w, wrate, wlk, wdrate = O.wfm_batch_audio(x, fs, off, bw, tau)
    assert (rate, drate) == (wrate, wdrate)
    assert lk == wlk
    if want_locked is not None:
        assert lk == want_locked
    assert a.size == w.size
    for c in (0, 1):
        assert rel_l2(a[c::2], w[c::2]) <= 1e-5, (c, rel_l2(a[c::2], w[c::2]))
    return a, lk


def test_batch_stereo_station_2p4msps(cuda):
    scene, _ = synth.plain_wfm_scene(block=262_144)
    x = np.concatenate([scene.next_block().numpy() for _ in range(4)])
    # 2.4 MS/s: decimation round(12.5) = 13 -> 184615 S/s, a 9600-arm resampler
    a, lk = _check(x, 2_400_000, 300_000.0, 250_000.0, 50.0, want_locked=True)
    assert not np.allclose(a[0::2], a[1::2])


def test_batch_noise_falls_back_to_mono(cuda):
    rng = np.random.default_rng(7)
    x = (0.1 * (rng.standard_normal(600_000) + 1j * rng.standard_normal(600_000))).astype(np.complex64)
    a, lk = _check(x, 2_400_000, -150_000.0, 200_000.0, 75.0, want_locked=False)
    assert np.array_equal(a[0::2], a[1::2])


def test_batch_192k_and_10msps(cuda):
    scene, _ = synth.plain_wfm_scene(block=262_144)
    x = scene.next_block().numpy()
    # 1.92 MS/s read as a station at DC: D 10 to exactly 192 kS/s, no shift, no de-emphasis
    _check(x, 1_920_000, 0.0, 180_000.0, 0.0)
    scene2, st = synth.fm_band_scene(block=1 << 20, n_stations=8, seconds=0.3)
    y = scene2.next_block().numpy()
    # 10 MS/s: D 52 -> 192307 S/s, a 48000-arm resampler
    _check(y, 10_000_000, st[3].offset_hz, 250_000.0, 50.0)


def test_batch_device_input_and_short(cuda):
    import torch
    scene, _ = synth.plain_wfm_scene(block=262_144)
    x = scene.next_block()
    a_dev = G.wfm_batch_audio(x.to("cuda"), 2_400_000, 300_000.0, 250_000.0)
    a_host = G.wfm_batch_audio(x.numpy(), 2_400_000, 300_000.0, 250_000.0)
    assert np.array_equal(a_dev[0], a_host[0]) and a_dev[1:] == a_host[1:]
    # fewer than two decimated samples: no audio, as the reference's nil
    e = G.wfm_batch_audio(x.numpy()[:13], 2_400_000, 300_000.0, 250_000.0)
    assert e[0].size == 0
    w = O.wfm_batch_audio(x.numpy()[:13], 2_400_000, 300_000.0, 250_000.0)
    assert w[0].size == 0
