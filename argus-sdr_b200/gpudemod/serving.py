"""Serving loop over the channel runner: continuous batching of demod requests.

The reference serves demod requests from its detector/tracker and from
`/api/demod` and `/ws/audio` (cmd/sdrd ws_handlers.go, helpers.go), each one
running its own per-signal extraction and CPU demod chain.  Here every request
becomes a slot of one `ChannelRunner`: its NCO phase, FIR/decimator history,
pilot PLL and RDS state stay resident on the device, requests arriving while
blocks are on the GPU join at the next block boundary once a slot and device
memory are free (the runner refuses admission beyond its device-memory
budget), and finished requests free their slot.  Every block runs all live
channels through one launch sequence; the loop records per-block latency
(runner events from the block's submit to its outputs in host memory) next to
throughput.

`poisson_requests` draws the request stream the serving benchmark describes:
Poisson arrivals, uniform-random frequency, a mode mix, log-uniform lifetimes.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import CH_AUDIO48K, CH_RDS, E_BUDGET, E_SLOTS, GPUDError, MODE_AM, MODE_CW, MODE_LSB, MODE_NFM, MODE_USB, \
    MODE_WFM_STEREO
from .synth import HEADROOM_FS, MODE_TABLE

RUNNER_MODE = {"WFM": MODE_WFM_STEREO, "NFM": MODE_NFM, "AM": MODE_AM, "USB": MODE_USB, "LSB": MODE_LSB,
               "CW": MODE_CW}


@dataclass
class Request:
    rid: int
    t_arrive: float   # seconds from the stream start
    t_end: float
    offset_hz: float
    kind: str         # WFM / NFM / AM / USB / LSB / CW
    out_rate: int = 0  # 0: the mode's rate (MODE_TABLE)
    taps: int = 0      # 0: the mode's tap count
    pcm: bool = True   # audio as 48 kHz s16le


def channel_spec(req: Request, pcm: bool = True):
    """(signal_id, offset, bandwidth, out_rate, taps, runner mode, flags) of a
    request: WFM as stereo with RDS; the narrow modes at their own rates; with
    `pcm` the audio comes back as the 48 kHz s16le stream /ws/audio sends."""
    out_rate, taps, bw = MODE_TABLE[req.kind]
    out_rate = req.out_rate or out_rate
    taps = req.taps or taps
    flags = (CH_RDS if req.kind == "WFM" else 0) | (CH_AUDIO48K if (pcm and req.pcm) else 0)
    return (req.rid, req.offset_hz, bw, out_rate, taps, RUNNER_MODE[req.kind], flags)


def poisson_requests(seed: int, seconds: float, rate_hz: float = 50.0, band_hz: float = 9_600_000.0,
                     mix=(("WFM", 0.30), ("NFM", 0.30), ("AM", 0.20), ("SSB", 0.15), ("CW", 0.05)),
                     life_s=(0.1, 30.0), warm_start: bool = True) -> list[Request]:
    """Requests over [0, seconds): Poisson arrivals at `rate_hz`, frequency
    uniform over +-band/2, mode drawn from `mix` (SSB split evenly USB/LSB),
    lifetime log-uniform over `life_s`.  With `warm_start`, arrivals are drawn
    from an earlier start so the stream opens at its steady-state population
    (Little's law: rate x mean lifetime)."""
    rng = np.random.default_rng(seed)
    t0 = -life_s[1] if warm_start else 0.0
    kinds = [k for k, _ in mix]
    probs = np.array([p for _, p in mix], dtype=np.float64)
    probs /= probs.sum()
    out, t, rid = [], t0, 1
    while True:
        t += rng.exponential(1.0 / rate_hz)
        if t >= seconds:
            break
        life = math.exp(rng.uniform(math.log(life_s[0]), math.log(life_s[1])))
        kind = kinds[rng.choice(len(kinds), p=probs)]
        if kind == "SSB":
            kind = "USB" if rng.random() < 0.5 else "LSB"
        off = float(rng.uniform(-band_hz / 2, band_hz / 2))
        if t + life > 0.0:
            out.append(Request(rid, max(t, 0.0), t + life, off, kind))
        rid += 1
    return out


def exact_divisors(n: int, lo: int, hi: int) -> list[int]:
    """Divisors of n in [lo, hi] (exact integer decimation ratios)."""
    return [d for d in range(lo, hi + 1) if n % d == 0]


# Headroom stress mix: the mixed batch's non-WFM ratios (NFM 40 : AM 30 :
# SSB 30 : CW 20) over 70 % of the channels and WFM (stereo + RDS) over 30 %,
# the serving stream's WFM share.
HEADROOM_MIX = (("WFM", 0.30), ("NFM", 0.70 * 40 / 120), ("AM", 0.70 * 30 / 120), ("SSB", 0.70 * 30 / 120),
                ("CW", 0.70 * 20 / 120))


class HeadroomMix:
    """Channel draws of the headroom stress: FIR lengths uniform over
    64..1024 taps, decimation log-uniform over the exact divisors of the
    sample rate in [16, 2400] (WFM at D = 192, 320 kS/s), WFM channels on a
    broadcast station (80 %) or anywhere, narrow channels on a narrow station
    (50 %) or anywhere.  Audio stays at the demod rate: several of these rates
    have no 48 kHz resampler of at most 128 arms."""

    def __init__(self, seed: int, wfm_offsets, narrow_stations, fs: int = HEADROOM_FS, t_lo: int = 64,
                 t_hi: int = 1024, d_lo: int = 16, d_hi: int = 2400, wfm_decim: int = 192):
        self.rng = np.random.default_rng(seed)
        self.fs = fs
        self.wfm = list(wfm_offsets)
        self.narrow = list(narrow_stations)
        self.divs = np.array(exact_divisors(fs, d_lo, d_hi), dtype=np.float64)
        self.t_lo, self.t_hi, self.wfm_decim = t_lo, t_hi, wfm_decim
        self.kinds = [k for k, _ in HEADROOM_MIX]
        p = np.array([q for _, q in HEADROOM_MIX])
        self.p = p / p.sum()
        self.rid = 0

    def decim(self) -> int:
        u = self.rng.uniform(math.log(self.divs[0]), math.log(self.divs[-1]))
        return int(self.divs[int(np.argmin(np.abs(np.log(self.divs) - u)))])

    def draw(self, t: float = 0.0) -> Request:
        rng = self.rng
        kind = self.kinds[rng.choice(len(self.kinds), p=self.p)]
        if kind == "SSB":
            kind = "USB" if rng.random() < 0.5 else "LSB"
        taps = int(rng.integers(self.t_lo, self.t_hi + 1))
        bw = MODE_TABLE[kind][2]
        edge = self.fs / 2 - bw
        if kind == "WFM":
            D = self.wfm_decim
            off = float(rng.choice(self.wfm)) if rng.random() < 0.8 else float(rng.uniform(-edge, edge))
        else:
            D = self.decim()
            near = [s for s in self.narrow if s.kind == kind]
            off = float(near[rng.integers(len(near))].offset_hz) if near and rng.random() < 0.5 \
                else float(rng.uniform(-edge, edge))
        self.rid += 1
        return Request(self.rid, t, math.inf, off, kind, out_rate=self.fs // D, taps=taps, pcm=False)


class ServingLoop:
    """Admits and retires requests at block boundaries and runs each block
    through every live channel."""

    def __init__(self, runner, block: int, sample_rate: int):
        self.r = runner
        self.block = block
        self.fs = sample_rate
        self.live = {}       # rid -> (slot, Request)
        self.pending = []    # requests not admitted yet (slots or memory busy)
        self.refused = set()  # requests refused admission at least once (slots or memory)
        self.admitted = 0
        self.retired = 0

    def _admit(self, req: Request):
        """True when admitted; otherwise the refusal code (E_BUDGET / E_SLOTS)."""
        try:
            slot = self.r.admit(*channel_spec(req))
        except GPUDError as e:
            if e.code in (E_BUDGET, E_SLOTS):
                return e.code
            raise
        self.live[req.rid] = (slot, req)
        self.admitted += 1
        return True

    def boundary(self, t_now: float, arrivals: list[Request]):
        """Block boundary at stream time t_now: retire finished requests, then
        admit waiting and newly arrived ones while slots and memory last."""
        for rid in [rid for rid, (_, q) in self.live.items() if q.t_end <= t_now]:
            slot, _ = self.live.pop(rid)
            self.r.retire(slot)
            self.retired += 1
        waiting = [q for q in self.pending if q.t_end > t_now] + list(arrivals)
        self.pending = []
        full = False
        for q in waiting:
            # no slot frees up before the next boundary once the cap is hit; a
            # budget refusal still lets a smaller channel through
            got = False if full else self._admit(q)
            if got is not True:
                full = full or got == E_SLOTS
                self.refused.add(q.rid)
                self.pending.append(q)

    def process(self, iq):
        """Run one block through every live channel (synchronous: outputs are
        in host memory on return)."""
        self.r.process_block(iq)
        return self.r.stats()

    @property
    def rejected(self) -> int:
        return len(self.refused)

    def channel_samples(self) -> int:
        return len(self.live) * self.block
