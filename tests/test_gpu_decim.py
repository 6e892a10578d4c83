"""Pre-demod decimation (gpud_channel_spec.demod_decim) on the GPU runner
against the oracle chain: extraction at out_rate, the stateful 101-tap
decimating low-pass (dsp/decimating_fir.go:6-95), then the demodulator at
out_rate / demod_decim (recorder/streamer.go:1098-1146)."""
import numpy as np
import pytest

import gpudemod as G
from gpudemod import synth
from oracle import oracle as O
from signals import rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _wfm_scene(block):
    """2.048 MS/s with one WFM station at +300 kHz: 512 kS/s extraction, the
    snip rate for which the reference forces decim1 = 2 (256 kS/s demod)."""
    rng = np.random.default_rng(synth.CONFIG_SEEDS[0])
    fs = 2_048_000
    st = synth.make_wfm_station(rng, 300_000.0, 1.0, seconds=12 * block / fs + 1)
    sigma = synth.noise_sigma_for_snr(1.0, 30.0, 200_000.0, fs)
    return synth.WidebandScene(fs, block, [st], sigma, synth.CONFIG_SEEDS[0], "cpu")


def _compare(g, w, ctx):
    assert g["n_iq"] == w["iq"].size, ctx
    if w["iq"].size:
        assert rel_l2(g["iq"], w["iq"]) <= TOL, ctx
    assert g["audio"].size == w["audio"].size, (ctx, g["audio"].size, w["audio"].size)
    if w["audio"].size:
        assert rel_l2(g["audio"], w["audio"]) <= TOL, (ctx, rel_l2(g["audio"], w["audio"]))
    assert g["rds"].size == w["rds"].size, ctx
    if w["rds"].size:
        assert rel_l2(g["rds"], w["rds"]) <= TOL, (ctx, rel_l2(g["rds"], w["rds"]))
    assert g["locked"] == w["locked"] and g["stereo"] == w["stereo"], ctx


def test_wfm_stereo_decim2_matches_oracle(cuda):
    block = 262_144
    scene = _wfm_scene(block)
    fs, rate = 2_048_000, 512_000
    r = G.ChannelRunner(fs, block, max_channels=2)
    slot = r.admit(1, 300_000.0, 250_000.0, rate, 128, G.MODE_WFM_STEREO, G.CH_RDS | G.CH_EMIT_IQ, demod_decim=2)
    oc = O.OracleChannel(fs, 300_000.0, 250_000.0, rate, 128, O.MODE_WFM_STEREO, rds=True, demod_decim=2)
    try:
        for b in range(10):
            # odd lengths: odd extraction counts move the decimator phase across blocks
            x = scene.next_block().numpy()[: block - 4 * 1021 * (b % 3) - 4 * (b & 1)]
            r.process_block(x)
            g = r.result(slot)
            assert g["rds_rate"] == 256_000 // 13
            _compare(g, oc.process(x), b)
    finally:
        r.close()


@pytest.mark.parametrize("kind,mode,rate,decim", [
    ("NFM", G.MODE_NFM, 50_000, 2), ("AM", G.MODE_AM, 100_000, 4),
    ("USB", G.MODE_USB, 25_000, 2), ("CW", G.MODE_CW, 10_000, 2)])
def test_narrow_modes_with_decim_match_oracle(cuda, kind, mode, rate, decim):
    fs, block = 10_000_000, 1 << 20
    scene, chans = synth.mixed_scene(device="cuda", block=block)
    off = next(o for k, o in chans if k == kind)
    _, taps, bw = synth.MODE_TABLE[kind]
    r = G.ChannelRunner(fs, block, max_channels=2)
    slot = r.admit(2, off, bw, rate, taps, mode, G.CH_EMIT_IQ, demod_decim=decim)
    oc = O.OracleChannel(fs, off, bw, rate, taps, mode, rds=False, demod_decim=decim)
    try:
        for b in range(3):
            x = scene.next_block().cpu().numpy()[: block - 40_961 * b]
            r.process_block(x)
            _compare(r.result(slot), oc.process(x), (kind, b))
    finally:
        r.close()


def test_decim_pcm_snapshot_and_pipelined(cuda):
    """48 kHz PCM from the 256 kS/s demod rate; the decimator's history and
    phase move with a snapshot; three blocks in flight equal one at a time."""
    block = 131_072
    scene = _wfm_scene(block)
    blocks = [scene.next_block().numpy()[: block - 4 * 333 * (k % 2)] for k in range(6)]
    spec = (1, 300_000.0, 250_000.0, 512_000, 128, G.MODE_WFM_STEREO, G.CH_RDS | G.CH_AUDIO48K)
    ra = G.ChannelRunner(2_048_000, block, max_channels=2)
    rb = G.ChannelRunner(2_048_000, block, max_channels=2)
    rp = G.ChannelRunner(2_048_000, block, max_channels=2)
    sa, sp = ra.admit(*spec, demod_decim=2), rp.admit(*spec, demod_decim=2)
    oc = O.OracleChannel(2_048_000, 300_000.0, 250_000.0, 512_000, 128, O.MODE_WFM_STEREO, demod_decim=2)
    back = O.Audio48(256_000, 2, wfm=True, deemph_us=50.0)
    try:
        seq = []
        for k, x in enumerate(blocks):
            ra.process_block(x)
            g = ra.result(sa)
            _, w_pcm = back.process(oc.process(x)["audio"])
            assert g["pcm"].size == w_pcm.size, k
            if w_pcm.size:
                d = np.abs(g["pcm"].astype(np.int32) - w_pcm.astype(np.int32))
                assert d.max() <= 1, (k, int(d.max()))
            seq.append((g["pcm"], g["rds"]))
            if k == 2:
                blob = ra.snapshot(sa)
                sb = rb.admit(*spec, demod_decim=2)
                rb.restore(sb, blob)
            if k >= 3:
                rb.process_block(x)
                h = rb.result(sb)
                assert np.array_equal(h["pcm"], seq[k][0]) and np.array_equal(h["rds"], seq[k][1])
        tickets, got = [], []
        for k, x in enumerate(blocks):
            tickets.append(rp.submit(x))
            if k >= 2:
                rp.wait(tickets[k - 2])
                got.append(rp.result(sp)["pcm"])
        for t in tickets[-2:]:
            rp.wait(t)
            got.append(rp.result(sp)["pcm"])
        for (a, _), b in zip(seq, got):
            assert np.array_equal(a, b)
    finally:
        ra.close()
        rb.close()
        rp.close()


def test_decim_rejects_bad_factor(cuda):
    r = G.ChannelRunner(2_048_000, 65_536, max_channels=2)
    try:
        with pytest.raises(G.GPUDError):
            r.admit(1, 0.0, 10_000.0, 32_000, 64, G.MODE_NFM, 0, demod_decim=65)
    finally:
        r.close()
