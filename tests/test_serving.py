"""Serving loop host logic (CPU): the request process and admission at block
boundaries, against a stand-in runner with a slot cap and a memory budget."""
import math

import numpy as np
import pytest

import gpudemod as G
from gpudemod import serving as SV


def test_poisson_requests_match_the_stream_description():
    reqs = SV.poisson_requests(1234, seconds=20.0, rate_hz=50.0)
    # arrivals inside the window: Poisson at 50/s
    inside = [q for q in reqs if q.t_arrive > 0.0]
    assert abs(len(inside) / 20.0 - 50.0) < 5.0
    # warm start: the population at any time is near rate x mean lifetime
    mean_life = (30.0 - 0.1) / math.log(30.0 / 0.1)
    for t in (0.0, 5.0, 10.0, 15.0):
        pop = sum(1 for q in reqs if q.t_arrive <= t < q.t_end)
        assert abs(pop - 50.0 * mean_life) < 0.25 * 50.0 * mean_life, (t, pop)
    kinds = [q.kind for q in inside]
    frac = {k: kinds.count(k) / len(kinds) for k in ("WFM", "NFM", "AM", "USB", "LSB", "CW")}
    assert abs(frac["WFM"] - 0.30) < 0.05 and abs(frac["NFM"] - 0.30) < 0.05
    assert abs(frac["AM"] - 0.20) < 0.05 and abs(frac["USB"] + frac["LSB"] - 0.15) < 0.04
    assert all(abs(q.offset_hz) <= 4_800_000.0 for q in reqs)
    lives = np.array([q.t_end - q.t_arrive for q in inside])
    assert lives.min() >= 0.1 - 1e-9 and lives.max() <= 30.0 + 1e-9
    assert SV.poisson_requests(1234, 20.0) == reqs  # seeded


class FakeRunner:
    """Slot cap and byte budget like gpud_runner_admit; WFM costs 3 units."""

    def __init__(self, cap, budget):
        self.cap, self.budget, self.used = cap, budget, 0
        self.slots = {}
        self.blocks = 0

    def admit(self, sid, off, bw, rate, taps, mode, flags):
        cost = 3 if mode == G.MODE_WFM_STEREO else 1
        if self.used + cost > self.budget:
            raise G.GPUDError(G.E_BUDGET, "budget")
        free = [s for s in range(self.cap) if s not in self.slots]
        if not free:
            raise G.GPUDError(G.E_SLOTS, "cap")
        self.slots[free[0]] = (sid, cost)
        self.used += cost
        return free[0]

    def retire(self, slot):
        _, cost = self.slots.pop(slot)
        self.used -= cost

    def process_block(self, iq):
        self.blocks += 1

    def stats(self):
        return {"active_channels": len(self.slots), "device_bytes_used": self.used}


def test_serving_loop_admits_retires_and_retries():
    r = FakeRunner(cap=6, budget=8)
    loop = SV.ServingLoop(r, 262144, 10_000_000)
    reqs = [SV.Request(i, 0.0, 0.05 * (i + 1), 1000.0 * i, k)
            for i, k in enumerate(["WFM", "WFM", "NFM", "AM", "CW", "USB", "LSB", "NFM"])]
    loop.boundary(0.0, reqs)
    # budget 8: WFM 3 + WFM 3 + NFM 1 + AM 1 -> the rest wait
    assert len(loop.live) == 4 and len(loop.pending) == 4 and r.used == 8
    loop.process(None)
    loop.boundary(0.06, [])  # request 0 ended at 0.05: its slot and 3 units free
    assert 0 not in loop.live and loop.retired == 1
    assert len(loop.live) == 6 and r.used <= 8
    # pending requests whose lifetime ended while waiting are dropped
    loop.boundary(1.0, [])
    assert not loop.live and not loop.pending and r.used == 0
    assert loop.admitted == loop.retired


def test_channel_spec_per_mode():
    for kind, (rate, taps, bw) in SV.MODE_TABLE.items():
        spec = SV.channel_spec(SV.Request(7, 0.0, 1.0, 12345.0, kind))
        assert spec[:5] == (7, 12345.0, bw, rate, taps)
        assert spec[5] == SV.RUNNER_MODE[kind]
        assert spec[6] == (G.CH_RDS if kind == "WFM" else 0) | G.CH_AUDIO48K
        assert SV.channel_spec(SV.Request(7, 0.0, 1.0, 0.0, kind), pcm=False)[6] & G.CH_AUDIO48K == 0
        assert 10_000_000 % rate == 0


def test_headroom_mix_draws():
    """Headroom stress channel draws: exact decimation ratios in [16, 2400]
    (WFM at 192), taps 64..1024, the 30 % WFM / mixed-batch ratio split, audio
    at the demod rate (no 48 kHz flag), RDS on every WFM channel."""
    from gpudemod import synth
    wfm = [-1.2e6, 0.4e6, 8.0e6]
    narrow = [synth.make_narrow_station(np.random.default_rng(1), k, 1e6 * i, 0.1)
              for i, k in enumerate(["NFM", "AM", "USB", "LSB", "CW"])]
    mix = SV.HeadroomMix(5, wfm, narrow)
    draws = [mix.draw() for _ in range(4000)]
    fs = synth.HEADROOM_FS
    kinds = {}
    for q in draws:
        kinds[q.kind] = kinds.get(q.kind, 0) + 1
        D = fs // q.out_rate
        assert fs % q.out_rate == 0 and D * q.out_rate == fs
        assert 16 <= D <= 2400
        assert 64 <= q.taps <= 1024
        assert abs(q.offset_hz) <= fs / 2
        spec = SV.channel_spec(q)
        assert spec[6] & G.CH_AUDIO48K == 0
        if q.kind == "WFM":
            assert D == 192 and spec[6] & G.CH_RDS
    n = len(draws)
    assert abs(kinds["WFM"] / n - 0.30) < 0.03
    assert abs(kinds["NFM"] / n - 0.7 * 40 / 120) < 0.03
    assert abs((kinds["USB"] + kinds["LSB"]) / n - 0.7 * 30 / 120) < 0.03
    # decimation spreads over the whole log range
    ds = np.array([fs // q.out_rate for q in draws if q.kind != "WFM"])
    assert ds.min() <= 20 and ds.max() >= 2000
    assert 0.3 < np.mean(np.log(ds) < np.log(196)) < 0.7
