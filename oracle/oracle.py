"""ctypes wrapper over oracle/liboracle.so -- the CPU restatement of the Argus
gpudemod path (see oracle.c for the per-function reference citations).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py, always as the checker or the timed
CPU baseline, never as the product.

Mirrors the reference's CPU oracle API: `CPUOracleRunner.StreamingExtract`
(gpudemod/streaming_oracle_extract.go:9-111), `ExactIntegerDecimation`,
`BuildPolyphaseTapsPhaseMajor`, `LowpassFIR`, the demodulators, the stateful
stereo decoder, the RDS baseband extractor and the RDS decoder.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

MODE_IQ, MODE_NFM, MODE_WFM, MODE_WFM_STEREO, MODE_AM, MODE_USB, MODE_LSB, MODE_CW = range(8)


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def _load() -> C.CDLL:
    if not os.path.exists(_LIB_PATH):
        build()
    lib = C.CDLL(_LIB_PATH)
    P = C.c_void_p
    i, d = C.c_int, C.c_double
    sig = {
        "or_lowpass_fir": (i, [d, i, i, P]),
        "or_exact_decim": (i, [i, i]),
        "or_polyphase_phase_len": (i, [i, i]),
        "or_build_polyphase": (i, [P, i, i, P]),
        "or_config_hash": (C.c_uint64, [C.c_int64, i, i, i]),
        "or_extract_host_core": (i, [P, i, i, d, P, P, i, i, P, P, P, i, P]),
        "or_extract_direct": (i, [P, i, d, P, P, i, i, P, P, P, P]),
        "or_extract_polyphase": (i, [P, i, d, P, P, i, i, P, P, P, i, P]),
        "or_fm_discrim": (i, [P, i, P]),
        "or_am_demod": (i, [P, i, P]),
        "or_ssb_demod": (i, [P, i, i, i, P]),
        "or_cw_demod": (i, [P, i, i, P]),
        "or_pll_coefficients": (None, [d, d, i, P, P]),
        "or_stereo_size": (C.c_size_t, []),
        "or_stereo_init": (None, [P]),
        "or_stereo_decode": (i, [P, P, i, i, P, P]),
        "or_wfm_stereo_stage": (i, [P, P, i, i, P, P, P]),
        "or_stereo_margins": (None, [P, P, P, P]),
        "or_rds_baseband_complex": (i, [P, i, i, P, P]),
        "or_rds_size": (C.c_size_t, []),
        "or_rds_init": (None, [P, i]),
        "or_rds_process": (i, [P, P, i, P]),
        "or_rds_syndrome": (C.c_uint16, [C.c_uint32]),
        "or_rds_dec_size": (C.c_size_t, []),
        "or_rds_dec_init": (None, [P]),
        "or_rds_decode": (i, [P, P, i, i]),
        "or_rds_dec_result": (None, [P, P, P, P]),
        "or_channel_size": (C.c_size_t, []),
        "or_channel_init": (i, [P, i, d, d, i, i, i, i]),
        "or_channel_process": (i, [P, P, i, P, P, P, P, P, P, P]),
        "or_channel_state": (None, [P, P, P, P]),
        "or_channel_stereo_margins": (None, [P, P, P, P]),
        "or_channel_set_offset": (None, [P, d]),
        "or_channel_set_demod_decim": (i, [P, i]),
        "or_nearest_exact_decimation_rate": (C.c_int64, [C.c_int64, C.c_int64, C.c_int64]),
        "or_snap_out_rate": (C.c_int64, [C.c_int64, C.c_int64]),
        "or_streaming_job": (i, [C.c_int64, d, d, d, i, i, d, P, P, P, P]),
        "or_batch_extract_job": (None, [C.c_int64, d, d, d, i, P, P, P]),
        "or_rds_job_out_rate": (C.c_int64, [C.c_int64]),
        "or_snippet_decim": (i, [C.c_int64, C.c_int64, i]),
        "or_shift_filter_decimate": (i, [P, i, i, d, P, i, i, P]),
        "or_engine_shift_filter_decimate": (i, [P, i, i, d, d, i, P, P]),
        "or_engine_size": (C.c_size_t, []),
        "or_engine_init": (None, [P, i]),
        "or_engine_demod": (i, [P, P, i, d, d, i, P, P]),
        "or_batch_slot": (i, [P, i, i, d, d, i, d, P, P, P]),
        "or_decim_fir_size": (C.c_size_t, []),
        "or_decim_fir_init": (i, [P, P, i, i]),
        "or_decim_fir_process": (i, [P, P, i, P]),
        "or_decim_fir_phase": (i, [P]),
        "or_resampler_size": (C.c_size_t, []),
        "or_resampler_init": (i, [P, i, i, i]),
        "or_resampler_init_any": (i, [P, i, i, i]),
        "or_resampler_release": (None, [P]),
        "or_resampler_ratio": (None, [P, P, P, P, P]),
        "or_resampler_bank": (None, [P, P]),
        "or_resampler_process": (i, [P, P, i, P]),
        "or_audio48_size": (C.c_size_t, []),
        "or_audio48_init": (i, [P, i, i, i, d]),
        "or_audio48_process": (i, [P, P, i, P, P]),
        "or_stereo_pilot": (i, [P, i, i, i, d, P, P, P, P]),
        "or_wfm_stereo_decode_batch": (i, [P, i, i, P, P, P, P]),
        "or_wfm_batch_audio": (i, [P, i, i, d, d, d, P, i, P, P, P]),
        "or_wfm_stereo_free": (i, [P, i, i, P]),
        "or_demod_audio_segment": (i, [i, P, i, i, d, d, P, i, P, P, P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_lib = _load()


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def _c64(x) -> np.ndarray:
    return np.ascontiguousarray(x, dtype=np.complex64)


def _f32(x) -> np.ndarray:
    return np.ascontiguousarray(x, dtype=np.float32)


# --------------------------------------------------------------------------
# dsp / gpudemod helpers
# --------------------------------------------------------------------------

def lowpass_fir(cutoff_hz: float, sample_rate: int, taps: int) -> np.ndarray:
    """dsp.LowpassFIR (internal/dsp/fir.go:6-28): odd length, float64."""
    out = np.zeros(taps + 2, dtype=np.float64)
    n = _lib.or_lowpass_fir(float(cutoff_hz), int(sample_rate), int(taps), _p(out))
    return out[:n].copy()


def exact_integer_decimation(sample_rate: int, out_rate: int) -> int:
    """gpudemod.ExactIntegerDecimation (cpu_oracle.go:155-163); raises on a
    non-integer ratio."""
    d = _lib.or_exact_decim(int(sample_rate), int(out_rate))
    if d <= 0:
        raise ValueError(f"streaming polyphase extractor requires integer decimation: "
                         f"sampleRate={sample_rate} outRate={out_rate}")
    return d


def build_polyphase_taps_phase_major(base, decim: int) -> np.ndarray:
    base = _f32(base)
    if decim <= 0 or base.size == 0:
        return np.zeros(0, dtype=np.float32)
    L = (base.size + decim - 1) // decim
    out = np.zeros(decim * L, dtype=np.float32)
    _lib.or_build_polyphase(_p(base), base.size, decim, _p(out))
    return out


def streaming_config_hash(signal_id: int, out_rate: int, num_taps: int, sample_rate: int) -> int:
    return int(_lib.or_config_hash(int(signal_id), int(out_rate), int(num_taps), int(sample_rate)))


def base_taps_f32(bandwidth: float, sample_rate: int, num_taps: int) -> np.ndarray:
    """Tap design of gpudemod/stream_state.go:57-77 (cutoff = max(BW/2, 200))."""
    cutoff = max(bandwidth / 2.0, 200.0)
    return lowpass_fir(cutoff, sample_rate, num_taps).astype(np.float32)


# --------------------------------------------------------------------------
# CPUOracleRunner (streaming_oracle_extract.go)
# --------------------------------------------------------------------------

@dataclass
class StreamingExtractJob:
    SignalID: int
    OffsetHz: float
    Bandwidth: float
    OutRate: int
    NumTaps: int
    ConfigHash: int


@dataclass
class StreamingExtractResult:
    SignalID: int
    IQ: np.ndarray
    Rate: int
    NOut: int
    PhaseCount: int
    HistoryLen: int


@dataclass
class CPUOracleState:
    SignalID: int
    ConfigHash: int = 0
    NCOPhase: float = 0.0
    Decim: int = 0
    PhaseCount: int = 0
    NumTaps: int = 0
    ShiftedHistory: np.ndarray = field(default_factory=lambda: np.zeros(0, np.complex64))
    BaseTaps: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))
    PolyphaseTaps: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))


def run_host_core(iq_new, sample_rate, offset_hz, phase, phase_count, num_taps, decim, history, poly):
    """runStreamingPolyphaseHostCore (streaming_host_core.go:5-64)."""
    iq = _c64(iq_new)
    poly = _f32(poly)
    keep = max(0, num_taps - 1)
    hist = np.zeros(max(keep, 1), dtype=np.complex64)
    h = _c64(history)
    hist[: h.size] = h
    hl = C.c_int(h.size)
    ph = C.c_double(phase)
    pc = C.c_int(phase_count)
    out = np.zeros(iq.size // max(1, decim) + 2, dtype=np.complex64)
    n = _lib.or_extract_host_core(_p(iq), iq.size, int(sample_rate), float(offset_hz), C.byref(ph),
                                  C.byref(pc), int(num_taps), int(decim), _p(hist), C.byref(hl),
                                  _p(poly), poly.size, _p(out))
    return out[:n].copy(), ph.value, pc.value, hist[: hl.value].copy()


class CPUOracleRunner:
    """gpudemod.CPUOracleRunner (streaming_oracle_extract.go:9-111)."""

    def __init__(self, sample_rate: int):
        self.SampleRate = sample_rate
        self.States: dict[int, CPUOracleState] = {}

    def ResetAllStates(self):
        self.States = {}

    def ResetSignalState(self, signal_id: int):
        self.States.pop(signal_id, None)

    def _get_or_init(self, job: StreamingExtractJob) -> CPUOracleState:
        decim = exact_integer_decimation(self.SampleRate, job.OutRate)
        st = self.States.get(job.SignalID)
        if st is None:
            st = CPUOracleState(SignalID=job.SignalID)
            self.States[job.SignalID] = st
        if st.ConfigHash != job.ConfigHash:  # ResetCPUOracleStateIfConfigChanged
            st.ConfigHash = job.ConfigHash
            st.NCOPhase = 0.0
            st.PhaseCount = 0
            st.ShiftedHistory = np.zeros(0, np.complex64)
        st.Decim = decim
        st.NumTaps = job.NumTaps if job.NumTaps > 0 else 101
        st.BaseTaps = base_taps_f32(job.Bandwidth, self.SampleRate, st.NumTaps)
        st.PolyphaseTaps = build_polyphase_taps_phase_major(st.BaseTaps, decim)
        return st

    def StreamingExtract(self, iq_new, jobs):
        results = []
        active = set()
        for job in jobs:
            active.add(job.SignalID)
            st = self._get_or_init(job)
            out, ph, pc, hist = run_host_core(iq_new, self.SampleRate, job.OffsetHz, st.NCOPhase,
                                              st.PhaseCount, st.NumTaps, st.Decim, st.ShiftedHistory,
                                              st.PolyphaseTaps)
            st.NCOPhase, st.PhaseCount, st.ShiftedHistory = ph, pc, hist
            results.append(StreamingExtractResult(job.SignalID, out, job.OutRate, out.size, pc, hist.size))
        for sid in list(self.States):
            if sid not in active:
                del self.States[sid]
        return results


def cpu_oracle_extract(iq, state: CPUOracleState, phase_inc: float, polyphase: bool = False) -> np.ndarray:
    """CPUOracleExtract / CPUOracleExtractPolyphase (cpu_oracle.go:32-130)."""
    iq = _c64(iq)
    keep = max(0, state.NumTaps - 1)
    hist = np.zeros(max(keep, 1), np.complex64)
    hist[: state.ShiftedHistory.size] = state.ShiftedHistory
    hl = C.c_int(state.ShiftedHistory.size)
    ph = C.c_double(state.NCOPhase)
    pc = C.c_int(state.PhaseCount)
    base = _f32(state.BaseTaps)
    out = np.zeros(iq.size // max(1, state.Decim) + 2, np.complex64)
    if polyphase:
        n = _lib.or_extract_polyphase(_p(iq), iq.size, float(phase_inc), C.byref(ph), C.byref(pc),
                                      state.NumTaps, state.Decim, _p(hist), C.byref(hl), _p(base),
                                      base.size, _p(out))
    else:
        n = _lib.or_extract_direct(_p(iq), iq.size, float(phase_inc), C.byref(ph), C.byref(pc),
                                   state.NumTaps, state.Decim, _p(hist), C.byref(hl), _p(base), _p(out))
    state.NCOPhase, state.PhaseCount = ph.value, pc.value
    state.ShiftedHistory = hist[: hl.value].copy()
    return out[:n].copy()


# --------------------------------------------------------------------------
# demodulators
# --------------------------------------------------------------------------

def fm_discrim(iq) -> np.ndarray:
    iq = _c64(iq)
    out = np.zeros(max(iq.size - 1, 1), np.float32)
    n = _lib.or_fm_discrim(_p(iq), iq.size, _p(out))
    return out[:n].copy()


def am_demod(iq) -> np.ndarray:
    iq = _c64(iq)
    out = np.zeros(max(iq.size, 1), np.float32)
    n = _lib.or_am_demod(_p(iq), iq.size, _p(out))
    return out[:n].copy()


def ssb_demod(iq, sample_rate: int, usb: bool) -> np.ndarray:
    iq = _c64(iq)
    out = np.zeros(max(iq.size, 1), np.float32)
    n = _lib.or_ssb_demod(_p(iq), iq.size, int(sample_rate), 1 if usb else 0, _p(out))
    return out[:n].copy()


def cw_demod(iq, sample_rate: int) -> np.ndarray:
    iq = _c64(iq)
    out = np.zeros(max(iq.size, 1), np.float32)
    n = _lib.or_cw_demod(_p(iq), iq.size, int(sample_rate), _p(out))
    return out[:n].copy()


def pll_coefficients(loop_bw: float, damping: float, sample_rate: int):
    a, b = C.c_double(), C.c_double()
    _lib.or_pll_coefficients(loop_bw, damping, sample_rate, C.byref(a), C.byref(b))
    return a.value, b.value


class StereoDecoder:
    """streamSession stereo state: stereoDecodeStateful + hysteresis + mono
    fallback filter (recorder/streamer.go:1355-1644)."""

    def __init__(self):
        self._buf = C.create_string_buffer(_lib.or_stereo_size())
        _lib.or_stereo_init(self._buf)

    def decode(self, mono, sample_rate):
        mono = _f32(mono)
        out = np.zeros(2 * max(mono.size, 1), np.float32)
        lk = C.c_int()
        n = _lib.or_stereo_decode(self._buf, _p(mono), mono.size, int(sample_rate), _p(out), C.byref(lk))
        return out[: 2 * n].copy(), bool(lk.value)

    def stage(self, mono, sample_rate):
        mono = _f32(mono)
        out = np.zeros(2 * max(mono.size, 1), np.float32)
        lk, en = C.c_int(), C.c_int()
        n = _lib.or_wfm_stereo_stage(self._buf, _p(mono), mono.size, int(sample_rate), _p(out),
                                     C.byref(lk), C.byref(en))
        return out[: 2 * n].copy(), bool(lk.value), bool(en.value)

    def margins(self):
        c, f, e = C.c_double(), C.c_double(), C.c_double()
        _lib.or_stereo_margins(self._buf, C.byref(c), C.byref(f), C.byref(e))
        return c.value, f.value, e.value


def rds_baseband_complex(iq, sample_rate: int):
    """demod.RDSBasebandComplex (internal/demod/fm.go:143-163)."""
    iq = _c64(iq)
    out = np.zeros(iq.size // max(1, sample_rate // 19000) + 2, np.complex64)
    rate = C.c_int()
    n = _lib.or_rds_baseband_complex(_p(iq), iq.size, int(sample_rate), _p(out), C.byref(rate))
    return out[:n].copy(), rate.value


class RDSStream:
    """Streaming RDS baseband over a discriminator stream (equal to one
    RDSBasebandComplex call over the concatenation)."""

    def __init__(self, sample_rate: int):
        self._buf = C.create_string_buffer(_lib.or_rds_size())
        _lib.or_rds_init(self._buf, int(sample_rate))
        self.dr = max(1, sample_rate // 19000)

    def process(self, disc) -> np.ndarray:
        disc = _f32(disc)
        out = np.zeros(disc.size // self.dr + 2, np.complex64)
        n = _lib.or_rds_process(self._buf, _p(disc), disc.size, _p(out))
        return out[:n].copy()


def rds_syndrome(raw: int) -> int:
    return int(_lib.or_rds_syndrome(raw & 0x3FFFFFF))


class RDSDecoder:
    """rds.Decoder (internal/rds/rds.go:78-636)."""

    def __init__(self):
        self._buf = C.create_string_buffer(_lib.or_rds_dec_size())
        _lib.or_rds_dec_init(self._buf)

    def decode(self, samples, sample_rate: int) -> int:
        s = _c64(samples)
        return int(_lib.or_rds_decode(self._buf, _p(s), s.size, int(sample_rate)))

    def result(self):
        pi = C.c_uint16()
        ps = C.create_string_buffer(9)
        rt = C.create_string_buffer(65)
        _lib.or_rds_dec_result(self._buf, C.byref(pi), ps, rt)
        return int(pi.value), ps.value.decode("ascii"), rt.value.decode("ascii")


# --------------------------------------------------------------------------
# per-channel block pipeline
# --------------------------------------------------------------------------

class DecimatingFIR:
    """StatefulDecimatingFIRComplex (dsp/decimating_fir.go:6-95): float64
    delay line and accumulation, one output whenever the phase counter is 0."""

    def __init__(self, taps, factor):
        t = np.ascontiguousarray(taps, dtype=np.float64)
        self._buf = C.create_string_buffer(_lib.or_decim_fir_size())
        if _lib.or_decim_fir_init(self._buf, t.ctypes.data, t.size, int(factor)) != 0:
            raise ValueError("1..128 taps")
        self.factor = max(1, int(factor))

    @property
    def phase(self):
        return _lib.or_decim_fir_phase(self._buf)

    def process(self, iq):
        x = _c64(iq)
        out = np.zeros(x.size + 1, np.complex64)
        n = _lib.or_decim_fir_process(self._buf, x.ctypes.data, x.size, out.ctypes.data)
        return out[:n]


class OracleChannel:
    """One channel's block-by-block chain (extract -> demod -> stereo -> RDS),
    see or_channel_process in oracle.c."""

    def __init__(self, sample_rate, offset_hz, bandwidth, out_rate, num_taps, mode, rds=True, demod_decim=1):
        self._buf = C.create_string_buffer(_lib.or_channel_size())
        rc = _lib.or_channel_init(self._buf, int(sample_rate), float(offset_hz), float(bandwidth),
                                  int(out_rate), int(num_taps), int(mode), 1 if rds else 0)
        if rc != 0:
            raise ValueError("non-integer decimation")
        _lib.or_channel_set_demod_decim(self._buf, int(demod_decim))
        self.decim = sample_rate // out_rate
        self.out_rate = out_rate // max(1, int(demod_decim))

    def process(self, block):
        x = _c64(block)
        cap = x.size // self.decim + 4
        iq = np.zeros(cap, np.complex64)
        audio = np.zeros(2 * cap, np.float32)
        rds = np.zeros(cap // max(1, self.out_rate // 19000) + 4, np.complex64)
        niq, na, nr, fl = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        _lib.or_channel_process(self._buf, _p(x), x.size, _p(iq), C.byref(niq), _p(audio), C.byref(na),
                                _p(rds), C.byref(nr), C.byref(fl))
        return {
            "iq": iq[: niq.value].copy(),
            "audio": audio[: na.value].copy(),
            "rds": rds[: nr.value].copy(),
            "locked": bool(fl.value & 1),
            "stereo": bool(fl.value & 2),
        }

    def state(self):
        ph, pc, hl = C.c_double(), C.c_int(), C.c_int()
        _lib.or_channel_state(self._buf, C.byref(ph), C.byref(pc), C.byref(hl))
        return ph.value, pc.value, hl.value

    def margins(self):
        c, f, e = C.c_double(), C.c_double(), C.c_double()
        _lib.or_channel_stereo_margins(self._buf, C.byref(c), C.byref(f), C.byref(e))
        return c.value, f.value, e.value

    def set_offset(self, offset_hz):
        _lib.or_channel_set_offset(self._buf, float(offset_hz))


class Resampler:
    """dsp.Resampler (internal/dsp/resample.go:45-153): rational polyphase
    resampler, stateful across Process calls."""

    def __init__(self, in_rate: int, out_rate: int, taps_per_phase: int = 32):
        self._buf = C.create_string_buffer(_lib.or_resampler_size())
        if _lib.or_resampler_init_any(self._buf, int(in_rate), int(out_rate), int(taps_per_phase)) != 0:
            raise ValueError("resampler bank too large")

    def __del__(self):
        if _lib is not None and getattr(self, "_buf", None) is not None:
            _lib.or_resampler_release(self._buf)

    def ratio(self):
        l, m, k, t = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        _lib.or_resampler_ratio(self._buf, C.byref(l), C.byref(m), C.byref(k), C.byref(t))
        return l.value, m.value, k.value, t.value

    def bank(self) -> np.ndarray:
        l, _, k, _ = self.ratio()
        out = np.zeros(l * k, np.float64)
        _lib.or_resampler_bank(self._buf, _p(out))
        return out.reshape(l, k)

    def process(self, x) -> np.ndarray:
        x = _f32(x)
        l, m, _, _ = self.ratio()
        out = np.zeros(int(x.size * l / m) + 8, np.float32)
        n = _lib.or_resampler_process(self._buf, _p(x), x.size, _p(out))
        return out[:n].copy()


class Audio48:
    """48 kHz audio back end of one channel (recorder/streamer.go:1408-1470,
    569-575): resample each audio channel to 48 kHz, de-emphasis and x0.35 for
    WFM, s16le encoding."""

    def __init__(self, in_rate: int, channels: int, wfm: bool, deemph_us: float = 50.0):
        self.channels = channels
        self.ratio = 48000.0 / in_rate
        self._buf = C.create_string_buffer(_lib.or_audio48_size())
        if _lib.or_audio48_init(self._buf, int(in_rate), int(channels), 1 if wfm else 0, float(deemph_us)) != 0:
            raise ValueError("resampler bank too large")

    def process(self, audio):
        a = _f32(audio)
        frames = a.size // self.channels
        cap = self.channels * (int(frames * self.ratio) + frames // 1000 + 64)
        f = np.zeros(cap, np.float32)
        pcm = np.zeros(cap, np.int16)
        n = _lib.or_audio48_process(self._buf, _p(a), frames, _p(f), _p(pcm))
        return f[:n].copy(), pcm[:n].copy()


def stereo_pilot(iq, sample_rate: int, window: bool = True, threshold: float = 4.0):
    """classifier.StereoPilotPresent (window=True) / estimateWFMPilot over the
    whole vector (window=False), internal/classifier/pll.go:75-131.  Returns
    (locked, ratio, best_hz, median, 201 magnitudes)."""
    x = _c64(iq)
    ratio, best, med = C.c_double(), C.c_double(), C.c_double()
    mags = np.zeros(201, np.float64)
    lk = _lib.or_stereo_pilot(_p(x), x.size, int(sample_rate), 1 if window else 0, float(threshold),
                              C.byref(ratio), C.byref(best), C.byref(med), _p(mags))
    return bool(lk), ratio.value, best.value, med.value, mags


def wfm_stereo_decode_batch(mono, sample_rate: int):
    """wfmStereoDecodeBatch (recorder/wfm_batch_stereo.go:74-155).  Returns
    (interleaved L/R float32, locked, pilot/total power ratio, loop Hz, mean
    |err|)."""
    m = np.ascontiguousarray(mono, dtype=np.float32)
    out = np.zeros(2 * m.size, np.float32)
    ratio, fhz, err = C.c_double(), C.c_double(), C.c_double()
    lk = _lib.or_wfm_stereo_decode_batch(_p(m), m.size, int(sample_rate), _p(out), C.byref(ratio), C.byref(fhz),
                                         C.byref(err))
    return out, bool(lk), ratio.value, fhz.value, err.value


def wfm_batch_audio(iq, sample_rate: int, offset_hz: float, bandwidth: float, deemph_us: float = 50.0):
    """demodWFMStereoBatchAudio (recorder/wfm_batch_stereo.go:10-72) over one
    capture.  Returns (interleaved float32 L/R audio, its rate, locked, demod
    rate)."""
    x = _c64(iq)
    cap = 2 * (int(x.size * 48000 / max(1, sample_rate)) + x.size // 4 + 256)
    out = np.zeros(cap, np.float32)
    orate, lk, drate = C.c_int(), C.c_int(), C.c_int()
    n = _lib.or_wfm_batch_audio(_p(x), x.size, int(sample_rate), float(offset_hz), float(bandwidth), float(deemph_us),
                                _p(out), cap, C.byref(orate), C.byref(lk), C.byref(drate))
    if n < 0:
        raise ValueError("batch audio: output capacity or resampler")
    return out[:n].copy(), orate.value, bool(lk.value), drate.value


def wfm_stereo_free(iq, sample_rate: int):
    """demod.wfmStereo (demod/fm.go:92-123): free-running 38 kHz stereo of one
    call.  Returns interleaved float32 L/R (2*(n-1))."""
    x = _c64(iq)
    out = np.zeros(2 * max(x.size, 1), np.float32)
    m = _lib.or_wfm_stereo_free(_p(x), x.size, int(sample_rate), _p(out))
    return out[: 2 * m].copy()


def demod_audio_segment(mode: int, iq, sample_rate: int, offset_hz: float, bandwidth: float):
    """demodAudioCPU (recorder/cpu_audio.go:10-75) over one segment.  Returns
    (audio float32, channels, audio rate, demod rate)."""
    x = _c64(iq)
    cap = 2 * x.size + 64
    out = np.zeros(cap, np.float32)
    ch, orate, drate = C.c_int(), C.c_int(), C.c_int()
    n = _lib.or_demod_audio_segment(int(mode), _p(x), x.size, int(sample_rate), float(offset_hz), float(bandwidth),
                                    _p(out), cap, C.byref(ch), C.byref(orate), C.byref(drate))
    if n < 0:
        raise ValueError("segment audio: output capacity")
    return out[:n].copy(), ch.value, orate.value, drate.value



# --------------------------------------------------------------------------
# surveillance spectrum (internal/fft): the published DFT in float64 (numpy's
# FFT), with the reference's window, scaling, floor and fftshift
# --------------------------------------------------------------------------

def hann(n: int) -> np.ndarray:
    """fftutil.Hann (fft.go:5-17)."""
    if n <= 1:
        return np.ones(max(n, 0))
    return 0.5 * (1 - np.cos(2 * np.pi * np.arange(n) / (n - 1)))


def spectrum(iq, window=None) -> np.ndarray:
    """fftutil.Spectrum (fft.go:19-55): 20 log10(|X|/n + 1e-12), DC at n/2."""
    x = np.asarray(iq, np.complex64).astype(np.complex128)
    n = x.size
    if n == 0:
        return np.zeros(0)
    if window is not None and len(window) == n:
        x = x * np.asarray(window, np.float64)
    mag = np.abs(np.fft.fft(x)) / n
    return np.roll(20 * np.log10(mag + 1e-12), n // 2)


def welch_psd(iq, seg: int, overlap: float, window=None) -> np.ndarray:
    """fftutil.WelchPSD (welch.go:15-66): mean |X|^2/n^2 over segments at
    step int(seg (1 - overlap)), 10 log10(. + 1e-24), DC at seg/2; fewer
    samples than a segment: Spectrum(iq, window)."""
    x = np.asarray(iq, np.complex64).astype(np.complex128)
    overlap = min(max(overlap, 0.0), 0.95)
    step = max(1, int(seg * (1 - overlap)))
    acc, segs = np.zeros(seg), 0
    w = np.asarray(window, np.float64) if window is not None and len(window) == seg else 1.0
    for start in range(0, x.size - seg + 1, step):
        mag = np.abs(np.fft.fft(x[start:start + seg] * w)) / seg
        acc += mag * mag
        segs += 1
    if segs == 0:
        return spectrum(iq, window)
    return np.roll(10 * np.log10(acc / segs + 1e-24), seg // 2)


# --------------------------------------------------------------------------
# job construction (cmd/sdrd): restated in oracle.c, wrapped here
# --------------------------------------------------------------------------
def nearest_exact_decimation_rate(sample_rate: int, target: int, min_rate: int) -> int:
    """cmd/sdrd/streaming_refactor.go:105-137."""
    return int(_lib.or_nearest_exact_decimation_rate(sample_rate, target, min_rate))


def snap_out_rate(sample_rate: int, target: int) -> int:
    """cmd/sdrd/helpers.go:292-310."""
    return int(_lib.or_snap_out_rate(sample_rate, target))


def streaming_job(sample_rate: int, tuner_center_hz: float, sig_center_hz: float, sig_bw_hz: float,
                  class_wfm: bool, fir_taps: int = 0, bw_mult: float = 0.0):
    """cmd/sdrd/streaming_refactor.go:16-60, one signal: (offset, bw, out_rate,
    taps), or None where the reference returns ExactIntegerDecimation's error."""
    off, bw, rate, taps = C.c_double(), C.c_double(), C.c_int64(), C.c_int()
    rc = _lib.or_streaming_job(sample_rate, tuner_center_hz, sig_center_hz, sig_bw_hz, int(class_wfm), fir_taps,
                               bw_mult, C.byref(off), C.byref(bw), C.byref(rate), C.byref(taps))
    return None if rc else (off.value, bw.value, int(rate.value), int(taps.value))


def batch_extract_job(sample_rate: int, tuner_center_hz: float, sig_center_hz: float, sig_bw_hz: float,
                      class_wfm: bool):
    """cmd/sdrd/helpers.go:174-194, one signal: (offset, bw, out_rate)."""
    off, bw, rate = C.c_double(), C.c_double(), C.c_int64()
    _lib.or_batch_extract_job(sample_rate, tuner_center_hz, sig_center_hz, sig_bw_hz, int(class_wfm), C.byref(off),
                              C.byref(bw), C.byref(rate))
    return off.value, bw.value, int(rate.value)


def rds_job_out_rate(ring_rate: int) -> int:
    """cmd/sdrd/pipeline_runtime.go:1094-1101."""
    return int(_lib.or_rds_job_out_rate(ring_rate))


def snippet_decim(snip_rate: int, demod_rate: int, wfm: bool) -> int:
    """recorder/streamer.go:1098-1113."""
    return int(_lib.or_snippet_decim(snip_rate, demod_rate, int(wfm)))


# --------------------------------------------------------------------------
# the single-signal Engine and the legacy GPU batch slot
# --------------------------------------------------------------------------
def engine_shift_filter_decimate(iq, sample_rate: int, offset_hz: float, bw: float, out_rate: int):
    """Engine.ShiftFilterDecimate (gpudemod.go:325-350): (IQ, rate)."""
    x = _c64(iq)
    out = np.zeros(x.size + 1, np.complex64)
    rate = C.c_int()
    n = _lib.or_engine_shift_filter_decimate(_p(x), x.size, sample_rate, offset_hz, bw, out_rate, _p(out),
                                             C.byref(rate))
    if n < 0:
        raise ValueError("invalid output sample rate")
    return out[:n], rate.value


class Engine:
    """Engine.Demod state (gpudemod.go:81-100): first-call FIR taps and the
    BFO phase.  mode is the DemodType (0 NFM .. 5 CW)."""

    def __init__(self, sample_rate: int):
        self._st = np.zeros(_lib.or_engine_size(), np.uint8)
        _lib.or_engine_init(_p(self._st), sample_rate)

    def demod(self, iq, offset_hz: float, bw: float, mode: int):
        x = _c64(iq)
        out = np.zeros(x.size + 1, np.float32)
        rate = C.c_int()
        n = _lib.or_engine_demod(_p(self._st), _p(x), x.size, offset_hz, bw, mode, _p(out), C.byref(rate))
        if n < 0:
            raise ValueError("unsupported demod type")
        return out[:n], rate.value


def batch_slot(iq, sample_rate: int, offset_hz: float, bw: float, out_rate: int, phase_start: float = 0.0):
    """One legacy GPU batch slot (batch_runner_windows.go:142-182):
    (IQ, rate, phase_end)."""
    x = _c64(iq)
    out = np.zeros(x.size + 1, np.complex64)
    rate, pe = C.c_int(), C.c_double()
    n = _lib.or_batch_slot(_p(x), x.size, sample_rate, offset_hz, bw, out_rate, phase_start, _p(out), C.byref(rate),
                           C.byref(pe))
    if n == -1:
        raise ValueError("non-integer decimation")
    if n == -2:
        raise ValueError("not enough output samples after decimation")
    return out[:n], rate.value, pe.value
