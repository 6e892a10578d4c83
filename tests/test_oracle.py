"""The CPU oracle pinned against the reference's own known-answer tests for
this path (each test names the reference test it restates).  CPU only."""
import math

import numpy as np
import pytest

from oracle import oracle as O
from signals import (chunks_of, make_deterministic_iq, make_lowpass_taps, max_abs)


def _state(decim=20, taps=65, phase=0.0):
    t = make_lowpass_taps(taps)
    return O.CPUOracleState(SignalID=1, ConfigHash=123, NCOPhase=phase, Decim=decim, PhaseCount=0,
                            NumTaps=taps, BaseTaps=t,
                            PolyphaseTaps=O.build_polyphase_taps_phase_major(t, decim))


def test_polyphase_layout_kat():
    # polyphase_test.go:5-22
    got = O.build_polyphase_taps_phase_major(np.arange(1, 8, dtype=np.float32), 3)
    assert got.tolist() == [1, 4, 7, 2, 5, 0, 3, 6, 0]


def test_exact_integer_decimation():
    # cpu_oracle_test.go:60-67
    assert O.exact_integer_decimation(4_000_000, 200_000) == 20
    with pytest.raises(ValueError):
        O.exact_integer_decimation(4_000_000, 192_000)


def _chunked(iq, sizes, phase_inc, polyphase):
    st = _state()
    return np.concatenate([O.cpu_oracle_extract(c, st, phase_inc, polyphase) for c in chunks_of(iq, sizes)])


def test_monolithic_vs_chunked_direct():
    # cpu_oracle_test.go:39-58
    iq = make_deterministic_iq(200_000)
    mono = O.cpu_oracle_extract(iq, _state(), 0.017)
    chunked = _chunked(iq, [4096, 5000, 8192, 27307], 0.017, False)
    assert mono.size == chunked.size == 200_000 // 20
    assert max_abs(mono, chunked) <= 1e-5


def test_direct_vs_polyphase():
    # cpu_oracle_test.go:69-89
    iq = make_deterministic_iq(50_000)
    direct = O.cpu_oracle_extract(iq, _state(), 0.017, polyphase=False)
    poly = O.cpu_oracle_extract(iq, _state(), 0.017, polyphase=True)
    assert max_abs(direct, poly) <= 1e-5


@pytest.mark.parametrize("n,inc,sizes", [
    (120_000, 0.013, [4096, 3000, 8192, 7777, 12000]),   # oracle_validation_test.go:5-45
    (150_000, 0.017, [4096, 5000, 8192, 27307]),          # test_harness_test.go:18-32
])
def test_monolithic_vs_chunked_polyphase(n, inc, sizes):
    iq = make_deterministic_iq(n)
    mono = O.cpu_oracle_extract(iq, _state(), inc, polyphase=True)
    chunked = _chunked(iq, sizes, inc, True)
    assert max_abs(mono, chunked) <= 1e-5


def test_host_core_matches_oracle_polyphase():
    # streaming_host_core_test.go:5-40
    iq = make_deterministic_iq(12_000)
    st = _state()
    want = O.cpu_oracle_extract(iq, st, 0.017, polyphase=True)
    s2 = _state()
    out, phase, pc, hist = O.run_host_core(iq, 4_000_000, -0.017 * 4_000_000 / (2 * 3.141592653589793), 0.0, 0,
                                           65, 20, np.zeros(0, np.complex64), s2.PolyphaseTaps)
    assert max_abs(out, want) <= 1e-5
    assert phase != 0 and 0 <= pc < 20 and hist.size > 0


def test_even_taps_apply_first_T_of_odd_design():
    # LowpassFIR bumps an even T to T+1 (dsp/fir.go:7-9) while the stream keeps
    # T-1 history (stream_state.go:78-82): the T+1-th tap never applies.
    fs, out_rate, T = 2_400_000, 300_000, 128
    base = O.base_taps_f32(250_000, fs, T)
    assert base.size == 129
    iq = make_deterministic_iq(4096)
    poly = O.build_polyphase_taps_phase_major(base, 8)
    got, *_ = O.run_host_core(iq, fs, 10_000.0, 0.0, 0, T, 8, np.zeros(0, np.complex64), poly)
    st = O.CPUOracleState(SignalID=1, Decim=8, NumTaps=T, BaseTaps=base[:T].copy())
    want = O.cpu_oracle_extract(iq, st, -2 * math.pi * 10_000.0 / fs)
    assert max_abs(got, want) <= 1e-6


def test_runner_prunes_and_resets():
    # state_reset_test.go / oracle_runner_test.go: hash change zeroes state,
    # vanished signals are pruned
    r = O.CPUOracleRunner(4_000_000)
    a = O.StreamingExtractJob(11, 12_500.0, 20_000.0, 200_000, 65, 1001)
    b = O.StreamingExtractJob(22, -18_750.0, 16_000.0, 100_000, 33, 2002)
    r.StreamingExtract(make_deterministic_iq(512), [a, b])
    assert set(r.States) == {11, 22}
    assert r.States[11].PhaseCount == 512 % 20 and r.States[11].ShiftedHistory.size == 64
    a2 = O.StreamingExtractJob(11, 12_500.0, 20_000.0, 200_000, 65, 1002)
    r.StreamingExtract(np.zeros(0, np.complex64), [a2])
    assert set(r.States) == {11}
    assert r.States[11].NCOPhase == 0.0 and r.States[11].PhaseCount == 0
    assert r.States[11].ShiftedHistory.size == 0


def test_config_hash_ignores_offset_and_bandwidth():
    from gpudemod import StreamingConfigHash
    h = O.streaming_config_hash(7, 200_000, 65, 4_000_000)
    assert h == StreamingConfigHash(7, 123.0, 9999.0, 200_000, 65, 4_000_000)
    assert h != O.streaming_config_hash(7, 200_000, 66, 4_000_000)


# ---------------------------------------------------------------------------
# RDS baseband: streaming == one plain call (fm_rds_test.go:10-35, byte exact)
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("sr", [200_000, 250_000, 240_000])
def test_rds_baseband_stream_equals_plain(sr):
    rng = np.random.default_rng(1)
    for n in [0, 1, 2, 17, 999, 4096]:
        iq = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
        want, rate = O.rds_baseband_complex(iq, sr)
        assert rate == (sr // (sr // 19000) if n >= 2 else 0)
        disc = O.fm_discrim(iq)
        st = O.RDSStream(sr)
        got = np.concatenate([st.process(c) for c in chunks_of(disc, [1, 16, 333, 0, 1000])]) \
            if disc.size else np.zeros(0, np.complex64)
        assert got.size == want.size
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_rds_syndrome_and_group_kat():
    from gpudemod import synth
    for off in (synth.OFF_A, synth.OFF_B, synth.OFF_C, synth.OFF_CP, synth.OFF_D):
        for data in (0, 1, 0xABCD, 0xFFFF, 0x1234):
            blk = synth.rds_block(data, off)
            assert O.rds_syndrome(blk) == off == synth.rds_syndrome(blk)
            assert blk >> 10 == data


def test_rds_encoder_decoder_kat():
    """Encoder -> BPSK baseband -> decoder: PI/PS/RT recovered bit-exactly."""
    from gpudemod import synth
    pi, ps, rt = 0xC0DE, "ARGUSB2K", "RADIOTEXT ON A B200 - SEEDED GROUP KAT 0123456789"
    bits = synth.rds_bits(synth.rds_groups(pi, ps, rt), 3000)
    sym = synth.rds_symbols(bits)
    fs = 20000.0
    t = np.arange(int(len(sym) / synth.RDS_BAUD * fs) - 40) / fs
    pos = t * synth.RDS_BAUD
    k = np.floor(pos).astype(int)
    c = 0.5 * (1 + np.cos(np.pi * (pos - k)))
    level = sym[k] * c + sym[k + 1] * (1 - c)
    x = (0.3 * level * np.exp(1j * 0.7)).astype(np.complex64)
    d = O.RDSDecoder()
    groups = d.decode(x, 20000)
    got_pi, got_ps, got_rt = d.result()
    assert groups >= 20
    assert (got_pi, got_ps, got_rt) == (pi, ps, rt.rstrip())


# ---------------------------------------------------------------------------
# stereo decoder properties (recorder/streamer_test.go, stereo_lock_test.go)
# ---------------------------------------------------------------------------
def _tone_mag(x, f, sr):
    n = np.arange(len(x))
    return abs(np.sum(x * np.exp(-2j * np.pi * f * n / sr))) * 2 / len(x)


def test_stereo_pilot_lock_and_separation():
    # streamer_test.go:8-67 (same composite: L-R on cos 38 kHz, pilot sin 19 kHz)
    sr, blk = 192_000, 4096
    dec = O.StereoDecoder()
    for b in range(10):
        t = (b * blk + np.arange(blk)) / sr
        l, r = np.sin(2 * np.pi * 440 * t), np.sin(2 * np.pi * 880 * t)
        comp = 0.5 * (l + r) + 0.5 * (l - r) * np.cos(2 * np.pi * 38000 * t) + 0.1 * np.sin(2 * np.pi * 19000 * t)
        out, locked = dec.decode(comp.astype(np.float32), sr)
    assert locked and out.size == 2 * blk
    L, R = out[0::2], out[1::2]
    l440, l880, r440, r880 = (_tone_mag(L, 440, sr), _tone_mag(L, 880, sr), _tone_mag(R, 440, sr),
                              _tone_mag(R, 880, sr))
    assert l440 >= 0.05 or l880 >= 0.05
    left_is_l = l440 >= l880 * 1.3 and r880 >= r440 * 1.3
    right_is_l = l880 >= l440 * 1.3 and r440 >= r880 * 1.3
    assert left_is_l or right_is_l


def _gen_mpx(n, sr, audio_amp, pilot_amp, t0):
    t = t0 + np.arange(n) / sr
    audio = audio_amp * np.sin(2 * np.pi * 1000 * t)
    pilot = pilot_amp * np.sin(2 * np.pi * 19000 * t)
    lr = 0.3 * audio_amp * np.sin(2 * np.pi * 2000 * t) * np.sin(2 * np.pi * 38000 * t)
    return (audio + pilot + lr).astype(np.float32), t0 + n / sr


def test_stereo_lock_holds_through_loud_audio():
    # stereo_lock_test.go:31-63
    sr, blk = 256_000, 4096
    dec = O.StereoDecoder()
    amps = [0.1] * 6 + [0.9, 0.15, 0.95, 0.1, 0.9, 0.95, 0.12, 0.9, 0.95, 0.9, 0.1, 0.95]
    t0, loud, loud_locked = 0.0, 0, 0
    for b, amp in enumerate(amps):
        mpx, t0 = _gen_mpx(blk, sr, amp, 0.08, t0)
        _, locked = dec.decode(mpx, sr)
        if b >= 6 and amp >= 0.8:
            loud += 1
            loud_locked += int(locked)
    assert loud > 0 and loud_locked == loud


def test_stereo_no_false_lock_on_noise():
    # stereo_lock_test.go:67-84 (seeded numpy noise stands in for Go math/rand)
    sr, blk = 256_000, 4096
    dec = O.StereoDecoder()
    rng = np.random.default_rng(1)
    for _ in range(15):
        _, locked = dec.decode((rng.standard_normal(blk) * 0.3).astype(np.float32), sr)
        assert not locked


def test_pll_coefficients():
    a, b = O.pll_coefficients(50, 0.707, 300_000)
    bl = 50 / 300_000
    th = bl / (0.707 + 0.25 / 0.707)
    d = 1 + 2 * 0.707 * th + th * th
    assert a == pytest.approx(4 * 0.707 * th / d, rel=1e-15)
    assert b == pytest.approx(4 * th * th / d, rel=1e-15)


def test_demod_semantics():
    iq = make_deterministic_iq(1000)
    am = O.am_demod(iq)
    mag = np.abs(iq.astype(np.complex128))
    assert np.allclose(am, (mag.astype(np.float32) - np.float32(mag.mean())), atol=1e-6)
    usb = O.ssb_demod(iq, 48000, True)
    ph = 2 * np.pi * 700 / 48000 * np.arange(1, 1001)
    assert np.allclose(usb, iq.real * np.cos(ph) - iq.imag * np.sin(ph), atol=1e-6)
    cw = O.cw_demod(iq, 48000)
    assert np.allclose(cw, iq.real * np.cos(ph), atol=1e-6)
    d = O.fm_discrim(iq)
    assert d.size == 999
    assert np.allclose(d, np.angle(iq[1:].astype(np.complex128) * np.conj(iq[:-1].astype(np.complex128))),
                       atol=1e-6)


def test_truth64_chain_agrees_with_oracle():
    """The float64 truth chain and the reference-precision restatement differ
    only by float32 rounding (pins the truth's sample timing, taps, PLL, lock
    and RDS stream)."""
    from gpudemod import synth
    from oracle import truth64 as T64
    scene, _ = synth.plain_wfm_scene(block=65_536)
    o = O.OracleChannel(2_400_000, 300_000.0, 250_000.0, 300_000, 128, O.MODE_WFM_STEREO, rds=True)
    t = T64.Truth64Channel(2_400_000, 300_000.0, 250_000.0, 300_000, 128, T64.MODE_WFM_STEREO, rds=True)
    for _ in range(3):
        x = scene.next_block().numpy()
        a, b = o.process(x), t.process(x)
        for key in ("iq", "audio", "rds"):
            assert a[key].size == b[key].size
            d = np.linalg.norm(a[key] - b[key]) / np.linalg.norm(b[key])
            assert d < 2e-6, (key, d)
        assert a["locked"] == b["locked"]


# --- 48 kHz audio back end: the reference's resample_test.go cases ----------

def test_resampler_ratio_kat():
    # TestResamplerRatio (resample_test.go:26-44) and the gcd cases (:8-24)
    for inr, outr, l, m in [(51200, 48000, 15, 16), (44100, 48000, 160, 147), (48000, 48000, 1, 1),
                            (96000, 48000, 1, 2), (312500, 48000, 96, 625), (300000, 48000, 4, 25)]:
        assert O.Resampler(inr, outr).ratio()[:2] == (l, m)
    assert math.gcd(48000, 200000) == 8000  # gcd KAT restated by the ratio above


def test_resampler_identity_and_output_length():
    # TestResamplerIdentity (:46-62)
    x = np.sin(2 * np.pi * 440 * np.arange(1000) / 48000).astype(np.float32)
    y = O.Resampler(48000, 48000).process(x)
    assert y.size == x.size and np.max(np.abs(y - x)) <= 1e-4
    # TestResamplerOutputLength (:64-88)
    for inr, outr, n in [(51200, 48000, 5120), (51200, 48000, 10240), (44100, 48000, 4410),
                         (96000, 48000, 9600), (200000, 48000, 20000), (312500, 48000, 32768)]:
        x = np.sin(2 * np.pi * 1000 * np.arange(n) / inr).astype(np.float32)
        y = O.Resampler(inr, outr).process(x)
        assert abs(y.size - n * outr / inr) <= 3


def test_resampler_stream_continuity():
    # TestResamplerStreamContinuity (:90-165): M-aligned chunks bit-exact,
    # arbitrary chunks within one sample per chunk
    inr, outr = 51200, 48000
    sig = np.sin(2 * np.pi * 1000 * np.arange(inr) / inr).astype(np.float32)
    one = O.Resampler(inr, outr).process(sig)
    r2 = O.Resampler(inr, outr)
    aligned = np.concatenate([r2.process(sig[i:i + 3200]) for i in range(0, sig.size, 3200)])
    assert np.array_equal(one, aligned)
    r3 = O.Resampler(inr, outr)
    ch = inr // 15
    arb = np.concatenate([r3.process(sig[i:i + ch]) for i in range(0, sig.size, ch)])
    assert abs(arb.size - one.size) <= (sig.size + ch - 1) // ch


def test_resampler_tone_and_stereo():
    # TestResamplerTonePreservation (:176-202)
    inr, outr = 51200, 48000
    x = np.sin(2 * np.pi * 1000 * np.arange(inr) / inr).astype(np.float32)
    y = O.Resampler(inr, outr).process(x)
    z = y[101:]
    crossings = np.count_nonzero((z[:-1] <= 0) & (z[1:] > 0) | (z[:-1] >= 0) & (z[1:] < 0))
    assert abs(crossings / 2.0 * outr / (y.size - 101) - 1000) <= 10
    # TestStereoResampler (:204-235) through the stereo back end (no de-emphasis)
    n = inr // 2
    st = np.empty(2 * n, np.float32)
    st[0::2] = np.sin(2 * np.pi * 440 * np.arange(n) / inr)
    st[1::2] = np.sin(2 * np.pi * 880 * np.arange(n) / inr)
    f, pcm = O.Audio48(inr, 2, wfm=False).process(st)
    assert abs(f.size // 2 - n * outr / inr) <= 3
    assert np.sum(np.abs(f[100:200:2])) > 0.1 and np.sum(np.abs(f[101:201:2])) > 0.1
    # s16le: int16(clip(s * 32767)), truncating
    assert np.array_equal(pcm, np.clip(f * np.float32(32767), -32768, 32767).astype(np.int16))


def test_audio48_deemphasis_and_gain():
    # WFM: de-emphasis y = a y + (1-a) x (tau 50 us at 48 kHz) then x0.35
    inr = 312_500
    x = (0.5 * np.sin(2 * np.pi * 1000 * np.arange(32768) / inr)).astype(np.float32)
    plain = O.Resampler(inr, 48000).process(x)
    f, _ = O.Audio48(inr, 1, wfm=True, deemph_us=50.0).process(x)
    a = math.exp(-1.0 / (48000 * 50e-6))
    y, ref = 0.0, np.empty(plain.size, np.float32)
    for i, v in enumerate(plain):
        y = a * y + (1 - a) * float(v)
        ref[i] = np.float32(y)
    assert np.array_equal(f, ref * np.float32(0.35))


def _rs_advance(L, M, t0, n):
    """The closed form the runner's host mirror uses for Resampler.Process:
    frames produced and the phase counter after n inputs from counter t0."""
    if n <= 0:
        return 0, t0
    if L == M:
        return n, t0
    cdiv = lambda a, b: -((-a) // b)
    A = cdiv((n + 1) * L - t0, M) - 1
    last = -1 if A < 0 else max(0, min(A, cdiv(n * L - t0, M)))
    c_last = (t0 + last * M) // L if last >= 0 else 0
    return last + 1, t0 + (last + 1) * M - n * L - (L if c_last < n else 0)


@pytest.mark.parametrize("in_rate", [312_500, 300_000, 25_000, 12_500, 5_000, 51_200, 44_100])
def test_resampler_closed_form_counts(in_rate):
    """The per-call output count and phase counter of Resampler.Process,
    including its exit inside the consume loop, follow the closed form for
    every chunk length (so each 48 kHz output can be computed independently)."""
    rng = np.random.default_rng(in_rate)
    r = O.Resampler(in_rate, 48000)
    L, M, _, t = r.ratio()
    for n in list(rng.integers(0, 9000, 40)) + [1, 2, 3, M, L, 32768]:
        got = r.process(rng.standard_normal(int(n)).astype(np.float32)).size
        want, t_next = _rs_advance(L, M, t, int(n))
        t = r.ratio()[3]
        assert (got, t) == (want, t_next), (n, got, want, t, t_next)


def test_wfm_pilot_detection_kat():
    """TestWFMPilotDetection (classifier/hard_rules_test.go:39-58): 2 s at
    192 kS/s of an FM carrier modulated by a 19 kHz pilot at 10 % of 75 kHz
    locks within 5 Hz; noise alone does not lock."""
    fs = 192_000
    i = np.arange(2 * fs)
    dev = 0.1 * np.sin(2 * np.pi * 19000 * i / fs) * 75000 / fs
    ph = np.cumsum(2 * np.pi * dev)
    iq = (np.cos(ph) + 1j * np.sin(ph)).astype(np.complex64)
    lk, ratio, best, _, _ = O.stereo_pilot(iq, fs, window=False)
    assert lk and abs(best - 19000.0) <= 5
    rng = np.random.default_rng(3)
    noise = (rng.standard_normal(fs) + 1j * rng.standard_normal(fs)).astype(np.complex64)
    assert not O.stereo_pilot(noise, fs)[0]
    assert not O.stereo_pilot(iq, 32_000)[0]  # below 40 kS/s: no decision


def _decim_input(n, a, b):
    i = np.arange(n)
    return (((i % a) - (a // 2)) / 8.0 + 1j * ((i % b) - (b // 2)) / 8.0).astype(np.complex64)


def test_decimating_fir_stream_continuity():
    """dsp/decimating_fir_test.go:8-38: chunks of 733 equal one call."""
    taps = O.lowpass_fir(90000, 512000, 101)
    x = _decim_input(8192, 17, 11)
    whole = O.DecimatingFIR(taps, 2).process(x)
    d = O.DecimatingFIR(taps, 2)
    chunked = np.concatenate([d.process(x[i:i + 733]) for i in range(0, x.size, 733)])
    assert whole.size == chunked.size == 4096
    assert np.array_equal(whole, chunked)


def test_decimating_fir_equals_filter_then_decimate():
    """dsp/decimating_fir_test.go:40-58: length of ApplyFIR + Decimate; with a
    zero start the stateful stage is that pipeline sample for sample."""
    taps = O.lowpass_fir(90000, 512000, 101)
    x = _decim_input(48640, 13, 7)
    for factor in (2, 3):
        out = O.DecimatingFIR(taps, factor).process(x)
        xr, xi = x.real.astype(np.float64), x.imag.astype(np.float64)
        fr = np.convolve(xr, taps)[: x.size]
        fi = np.convolve(xi, taps)[: x.size]
        want = (fr[::factor].astype(np.float32) + 1j * fi[::factor].astype(np.float32)).astype(np.complex64)
        assert out.size == len(range(0, x.size, factor))
        # numpy's convolution sums in another order: a float32 rounding apart
        assert np.max(np.abs(out - want)) <= 1e-6


def test_decimating_fir_phase_carry():
    """The phase counter carried across calls: after n inputs from phase p the
    emitted count is ceil((n - p) / factor) and the new phase (p - n) mod factor."""
    taps = O.lowpass_fir(90000, 512000, 101)
    d = O.DecimatingFIR(taps, 3)
    p = 0
    for n in (1, 2, 5, 7, 100, 3, 4):
        out = d.process(_decim_input(n, 5, 3))
        want = (n - 1 - p) // 3 + 1 if n > p else 0
        assert out.size == want
        p = (p - n) % 3
        assert d.phase == p


def test_channel_demod_decim_halves_the_demod_rate():
    """recorder/streamer.go:1098-1146: WFM at 512 kS/s extraction, decim1 2,
    demodulator and stereo decoder at 256 kS/s."""
    fs, rate = 2_048_000, 512_000
    t = np.arange(1 << 16) / fs
    x = np.exp(2j * np.pi * 300e3 * t).astype(np.complex64)
    a = O.OracleChannel(fs, 300e3, 250e3, rate, 64, O.MODE_WFM_STEREO, rds=False, demod_decim=2)
    b = O.OracleChannel(fs, 300e3, 250e3, rate, 64, O.MODE_WFM_STEREO, rds=False)
    ra, rb = a.process(x), b.process(x)
    assert ra["iq"].size == rb["iq"].size == x.size // 4
    # first block: no discriminator bridge, one sample fewer at each rate
    assert ra["audio"].size == 2 * (ra["iq"].size // 2 - 1)
    assert rb["audio"].size == 2 * (rb["iq"].size - 1)
    assert a.out_rate == 256_000


def _wfm_capture(n_blocks=4):
    import sys, os
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "argus-sdr_b200"))
    from gpudemod import synth
    scene, _ = synth.plain_wfm_scene(block=262_144)
    return np.concatenate([scene.next_block().numpy() for _ in range(n_blocks)])


def test_batch_stereo_decoder_equals_one_streaming_call():
    """wfmStereoDecodeBatch and stereoDecodeStateful share their filters and
    pilot loop (recorder/wfm_batch_stereo.go:74-145, streamer.go:1525-1644):
    from a fresh state one streaming call yields the same L/R samples; only
    the lock rule differs (pilot/total power ratio instead of coherence)."""
    rng = np.random.default_rng(3)
    rate, n = 192_000, 40_000
    t = np.arange(n) / rate
    mono = (0.3 * np.sin(2 * np.pi * 1000 * t) + 0.1 * np.sin(2 * np.pi * 19000 * t)
            + 0.2 * np.sin(2 * np.pi * 38000 * t) * np.sin(2 * np.pi * 3000 * t)
            + 0.01 * rng.standard_normal(n)).astype(np.float32)
    batch, lk, ratio, fhz, err = O.wfm_stereo_decode_batch(mono, rate)
    stream, _ = O.StereoDecoder().decode(mono, rate)
    assert np.array_equal(batch, stream)
    assert lk and ratio > 0.003 and abs(fhz - 19000) < 250 and err < 0.35


def test_batch_audio_lock_rates_and_mono_fallback():
    """demodWFMStereoBatchAudio (recorder/wfm_batch_stereo.go:10-72): 2.4 MS/s
    decimates by round(12.5) = 13 to 184615 S/s and resamples to 48 kHz; a
    stereo station locks, noise does not and yields duplicated mono."""
    x = _wfm_capture()
    a, rate, lk, drate = O.wfm_batch_audio(x, 2_400_000, 300_000.0, 250_000.0)
    assert drate == 2_400_000 // 13 and rate == 48_000 and lk
    nm = (x.size + 12) // 13 - 1
    rs = O.Resampler(drate, 48_000)
    assert a.size == 2 * rs.process(np.zeros(nm, np.float32)).size
    assert not np.allclose(a[0::2], a[1::2])
    nz = (np.random.default_rng(1).standard_normal(x.size) + 1j * np.random.default_rng(2).standard_normal(x.size))
    b, rate2, lk2, _ = O.wfm_batch_audio((0.1 * nz).astype(np.complex64), 2_400_000, 300_000.0, 250_000.0)
    assert not lk2 and np.array_equal(b[0::2], b[1::2])
    # 1.92 MS/s: D 10 to exactly 192 kS/s; zero offset skips the shift
    c, rate3, _, drate3 = O.wfm_batch_audio(x[:200_000], 1_920_000, 0.0, 100_000.0, deemph_us=0.0)
    assert drate3 == 192_000 and rate3 == 48_000 and c.size > 0


def test_free_running_stereo_matches_float64_model():
    """demod.wfmStereo (demod/fm.go:92-123) against a float64 numpy model of
    the same steps: discriminator, 15 kHz L+R, 53k-23k band times
    2 cos((q+1) inc) through the 15 kHz filter (the L-R path carries the band
    filter's extra 50-sample delay, as the reference does), L/R matrix."""
    rate, n = 192_000, 30_000
    q = np.arange(n)
    left = 0.4 * np.sin(2 * np.pi * 1000 * q / rate)
    c = 0.5 * left + 0.5 * left * np.cos(2 * np.pi * 38000 * (q + 1) / rate)
    x = np.exp(1j * np.cumsum(np.concatenate([[0.0], 0.5 * c]))).astype(np.complex64)
    out = O.wfm_stereo_free(x, rate)
    assert out.size == 2 * n
    disc = np.angle(x[1:].astype(np.complex128) * np.conj(x[:-1].astype(np.complex128)))
    f = lambda s, h: np.convolve(s, h)[: s.size]
    lp = O.lowpass_fir(15000, rate, 101)
    lpr = f(disc, lp)
    bpf = f(disc, O.lowpass_fir(53000, rate, 101)) - f(disc, O.lowpass_fir(23000, rate, 101))
    lr = f(bpf * 2 * np.cos(2 * np.pi * 38000 * (q + 1) / rate), lp)
    assert np.linalg.norm(out[0::2] - 0.5 * (lpr + lr)) <= 1e-5 * np.linalg.norm(lpr)
    assert np.linalg.norm(out[1::2] - 0.5 * (lpr - lr)) <= 1e-5 * np.linalg.norm(lpr)


def test_segment_rates_and_second_stage():
    """demodAudioCPU (recorder/cpu_audio.go:10-75): decimation round(fs/48000)
    or round(fs/192000), anti-alias stage only above 48 kHz, stereo keeps whole
    frames."""
    rng = np.random.default_rng(4)
    x = (0.2 * (rng.standard_normal(240_000) + 1j * rng.standard_normal(240_000))).astype(np.complex64)
    a, ch, rate, drate = O.demod_audio_segment(O.MODE_NFM, x, 2_400_000, 1e5, 12_500.0)
    assert (ch, drate, rate) == (1, 48_000, 48_000) and a.size == 240_000 // 50 - 1
    b, ch, rate, drate = O.demod_audio_segment(O.MODE_WFM_STEREO, x, 2_400_000, 0.0, 200_000.0)
    frames = (240_000 + 12) // 13 - 1
    assert (ch, drate, rate) == (2, 184_615, 46_153) and b.size == 2 * (frames // 4)
    c, ch, rate, drate = O.demod_audio_segment(O.MODE_AM, x, 2_400_000, 0.0, 10_000.0)
    assert abs(np.mean(c)) < 1e-3  # per-call mean removed


def test_welch_reduces_noise_variance_and_keeps_peaks():
    """fft/welch_test.go:29-74: 16 half-overlapping Hann segments of 4096
    cut the noise floor's spread to under 0.6x a single periodogram's, and a
    signal at DC stays >= 10 dB above the median."""
    n, k = 4096, 16
    rng = np.random.default_rng(5)
    noise = (rng.standard_normal(n * k) + 1j * rng.standard_normal(n * k)).astype(np.complex64)
    single = O.spectrum(noise[:n], O.hann(n))
    welch = O.welch_psd(noise, n, 0.5, O.hann(n))
    assert np.std(welch) < 0.6 * np.std(single)
    t = np.arange(n * k)
    sig = (noise + 0.3 * np.exp(2j * np.pi * 1.5e3 * t / 2.5e6)).astype(np.complex64)
    w = O.welch_psd(sig, n, 0.5, O.hann(n))
    assert w[n // 2 - 20:n // 2 + 21].max() - np.median(w) >= 10
    # fftshift and scaling: a unit tone at bin 7 reads 0 dB at index n/2 + 7
    tone = np.exp(2j * np.pi * 7 * np.arange(n) / n).astype(np.complex64)
    s = O.spectrum(tone)
    assert abs(s[n // 2 + 7]) < 1e-6 and s.argmax() == n // 2 + 7  # complex64 samples: ~1e-8 dB
