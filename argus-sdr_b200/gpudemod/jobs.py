"""Job construction: how detected signals and demod requests become extraction
jobs for the runner (the reference's `cmd/sdrd` rules).  These rules decide
which (output rate, taps, bandwidth) classes the extractor sees in
production, and with them which channels share a decimation class.

- `build_streaming_jobs` -- buildStreamingJobs (cmd/sdrd/streaming_refactor.go:16-60)
- `nearest_exact_decimation_rate` -- streaming_refactor.go:105-137
- `snap_out_rate` -- cmd/sdrd/helpers.go:292-310
- `batch_extract_jobs` -- the ExtractJobs of extractSignalIQBatch (helpers.go:174-194)
- `rds_extract_job` -- the RDS job of the pipeline (pipeline_runtime.go:1094-1101,
  run by extractionManager.extractRDS, helpers.go:122-160)
- `snippet_decim` -- processSnippet's pre-demod decimation (recorder/streamer.go:1098-1113)
- `production_channel` -- the runner channel a streamed signal becomes: its
  streaming job plus the pre-demod decimation to the demodulator's rate.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

from . import (CH_AUDIO48K, CH_RDS, MODE_AM, MODE_CW, MODE_LSB, MODE_NFM, MODE_USB, MODE_WFM, MODE_WFM_STEREO,
               ExactIntegerDecimation, ExtractJob, StreamingConfigHash, StreamingExtractJob)

WFM_STREAM_OUT_RATE = 512_000   # helpers.go:279
WFM_STREAM_MIN_BW = 250_000.0   # helpers.go:280
NARROW_TARGET_RATE = 200_000    # streaming_refactor.go:43, helpers.go:168
NARROW_MIN_RATE = 128_000       # streaming_refactor.go:43
NARROW_MIN_BW = 20_000.0        # streaming_refactor.go:44-46
RDS_JOB_BW = 200_000.0          # pipeline_runtime.go:1101
RDS_TARGET_RATE = 250_000       # pipeline_runtime.go:1094

# OutputSampleRate of each demodulator (demod/fm.go:19-23, am.go:8, ssb.go:11-12, cw.go:8)
DEMOD_RATE = {"NFM": 48_000, "WFM": 192_000, "WFM_STEREO": 192_000, "AM": 48_000, "USB": 48_000, "LSB": 48_000,
              "CW": 48_000}
RUNNER_MODE = {"NFM": MODE_NFM, "WFM": MODE_WFM, "WFM_STEREO": MODE_WFM_STEREO, "AM": MODE_AM, "USB": MODE_USB,
               "LSB": MODE_LSB, "CW": MODE_CW}


@dataclass
class Signal:
    """The fields of detector.Signal the job builders read: ID, centre and
    bandwidth in Hz, and the classifier's modulation verdict ("" when
    unclassified)."""
    ID: int
    CenterHz: float
    BWHz: float
    ModType: str = ""


@dataclass
class ExtractionConfig:
    """extractionConfig (helpers.go:271-275): FIR taps (<= 0: 101) and the
    extraction bandwidth multiplier (<= 0: 1)."""
    firTaps: int = 0
    bwMult: float = 0.0


def is_wfm(sig: Signal) -> bool:
    """Broadcast-band centre (87.5-108 MHz) or a WFM classification
    (streaming_refactor.go:27-28, helpers.go:178)."""
    mhz = sig.CenterHz / 1e6
    return (87.5 <= mhz <= 108.0) or sig.ModType in ("WFM", "WFM_STEREO")


def nearest_exact_decimation_rate(sample_rate: int, target_rate: int, min_rate: int) -> int:
    """streaming_refactor.go:105-137: the target when it divides the sample
    rate; otherwise, over decimations floor(sr/target) +- 2 (at least 1), the
    exact rate sr/d >= min_rate closest to the target (the first of equal
    distances); the target itself when none qualifies (ExactIntegerDecimation
    then reports the error)."""
    if sample_rate <= 0 or target_rate <= 0:
        return target_rate
    if sample_rate % target_rate == 0:
        return target_rate
    td = sample_rate // target_rate
    best, best_dist = 0, sample_rate
    for d in range(max(1, td - 2), td + 3):
        rate = sample_rate // d
        if rate < min_rate or sample_rate % rate != 0:
            continue
        dist = abs(target_rate - rate)
        if dist < best_dist:
            best, best_dist = rate, dist
    return best if best > 0 else target_rate


def snap_out_rate(sample_rate: int, target: int) -> int:
    """helpers.go:292-310: sr / d for the divisor d <= 256 of the sample rate
    closest to sr / target (float64 distance, the first of equals)."""
    if sample_rate <= 0 or target <= 0:
        return target
    ideal = sample_rate / target
    best_d, best_err = 0, math.inf
    for d in range(1, min(256, sample_rate) + 1):
        if sample_rate % d:
            continue
        e = abs(d - ideal)
        if e < best_err:
            best_d, best_err = d, e
    return sample_rate // best_d if best_d >= 1 else target


def build_streaming_jobs(sample_rate: int, center_hz: float, signals, cfg: ExtractionConfig | None = None):
    """buildStreamingJobs (streaming_refactor.go:16-60): per signal, bandwidth
    x bwMult; WFM at 512 kS/s with at least 250 kHz, other signals at the
    exact rate nearest 200 kS/s (>= 128 kS/s) with at least 20 kHz; taps
    firTaps; offset from the tuner centre; ConfigHash over (id, out rate,
    taps, sample rate).  Raises ValueError, as the reference returns an
    error for the whole batch, when an out rate does not divide the sample
    rate."""
    cfg = cfg or ExtractionConfig()
    bw_mult = cfg.bwMult if cfg.bwMult > 0 else 1.0
    taps = cfg.firTaps if cfg.firTaps > 0 else 101
    jobs = []
    for sig in signals:
        bw = sig.BWHz * bw_mult
        if is_wfm(sig):
            out_rate = WFM_STREAM_OUT_RATE
            bw = max(bw, WFM_STREAM_MIN_BW)
        else:
            out_rate = nearest_exact_decimation_rate(sample_rate, NARROW_TARGET_RATE, NARROW_MIN_RATE)
            bw = max(bw, NARROW_MIN_BW)
        ExactIntegerDecimation(sample_rate, out_rate)
        off = sig.CenterHz - center_hz
        jobs.append(StreamingExtractJob(sig.ID, off, bw, out_rate, taps,
                                        StreamingConfigHash(sig.ID, off, bw, out_rate, taps, sample_rate)))
    return jobs


def batch_extract_jobs(sample_rate: int, center_hz: float, signals):
    """The ExtractJobs extractSignalIQBatch hands the batch runner
    (helpers.go:174-194): WFM snapped near 512 kS/s with at least 250 kHz,
    other signals snapped near 200 kS/s with at least 20 kHz, no bandwidth
    multiplier."""
    jobs = []
    for sig in signals:
        wfm = is_wfm(sig)
        bw = max(sig.BWHz, WFM_STREAM_MIN_BW if wfm else NARROW_MIN_BW)
        rate = snap_out_rate(sample_rate, WFM_STREAM_OUT_RATE if wfm else NARROW_TARGET_RATE)
        jobs.append(ExtractJob(sig.CenterHz - center_hz, bw, rate))
    return jobs


def rds_extract_job(ring_rate: int, offset_hz: float) -> ExtractJob:
    """The RDS window's extraction job (pipeline_runtime.go:1094-1101): out
    rate ring / max(1, floor(ring / 250000)), bandwidth 200 kHz."""
    d = max(1, ring_rate // RDS_TARGET_RATE)
    return ExtractJob(offset_hz, RDS_JOB_BW, ring_rate // d)


def snippet_decim(snip_rate: int, mode: str) -> int:
    """processSnippet's decim1 (streamer.go:1098-1113): round(snip rate /
    demodulator rate), at least 1; WFM forced to 2 when larger and the snip
    Nyquist reaches 200 kHz."""
    wfm = mode in ("WFM", "WFM_STEREO")
    x = snip_rate / DEMOD_RATE[mode]
    d = math.floor(x)
    if x - d >= 0.5:  # math.Round: half away from zero (x > 0; x - floor(x) is exact)
        d += 1
    d = max(1, int(d))
    if wfm and d > 2 and snip_rate // 2 >= 200_000:
        d = 2
    return d


def production_channel(job: StreamingExtractJob, mode: str, rds: bool = False, pcm: bool = False):
    """ChannelRunner.admit arguments of a streamed signal as production runs
    it: the streaming job's extraction, then processSnippet's stateful
    pre-demod decimation to the demodulator's rate (`demod_decim`), then the
    mode's demodulator (WFM_STEREO: stereo decoder, with RDS when asked)."""
    flags = (CH_RDS if (rds and mode in ("WFM", "WFM_STEREO")) else 0) | (CH_AUDIO48K if pcm else 0)
    return dict(signal_id=job.SignalID, offset_hz=job.OffsetHz, bandwidth=job.Bandwidth, out_rate=job.OutRate,
                num_taps=job.NumTaps, mode=RUNNER_MODE[mode], flags=flags, config_hash=job.ConfigHash,
                demod_decim=snippet_decim(job.OutRate, mode))
