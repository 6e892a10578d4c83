"""Seeded synthetic wideband IQ scenes for the gpudemod path.

The reference measures this path on live captures that are not part of its
tree; these seeded scenes stand in for them with the shapes the benchmark
configurations describe: FM broadcast stations with a stereo multiplex (L+R
program tones, 19 kHz pilot, L-R DSB-SC on 38 kHz, RDS BPSK on 57 kHz at
1187.5 bit/s carrying PI/PS/RT groups), NFM / AM / SSB / CW channels, and
complex AWGN.

Everything is built with torch so the same code generates a few blocks on the
CPU for the tests and gigabytes directly in HBM for the benchmark.  Phases are
accumulated in float64.

RDS framing follows the decoder of the reference (internal/rds/rds.go): 26-bit
blocks whose 10-bit check word satisfies `crcSyndrome(raw) == offset` for that
decoder's syndrome map (rds.go:590-599, a linear map over GF(2)), offset words
A 0x0FC, B 0x198, C 0x168, C' 0x350, D 0x1B4 (rds.go:509-515), differential
encoding (rds.go:196-215) and BPSK symbols at 1187.5 Bd (rds.go:98).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch

OFF_A, OFF_B, OFF_C, OFF_CP, OFF_D = 0x0FC, 0x198, 0x168, 0x350, 0x1B4
RDS_BAUD = 1187.5
PILOT_HZ = 19000.0


# --------------------------------------------------------------------------
# RDS group encoder
# --------------------------------------------------------------------------

def rds_syndrome(raw: int) -> int:
    """The decoder's syndrome map (restated; rds.go:590-599)."""
    poly = 0x1B9
    reg = raw & 0x3FFFFFF
    for i in range(25, 9, -1):
        if (reg >> i) & 1:
            reg ^= poly << (i - 10)
    return reg & 0x3FF


def rds_block(data: int, offset: int) -> int:
    """26-bit block whose syndrome under the decoder's map equals `offset`.
    The map is linear and the identity on the low 10 bits, so the check word
    is syndrome(data << 10) xor offset."""
    data &= 0xFFFF
    return (data << 10) | (rds_syndrome(data << 10) ^ offset)


def rds_groups(pi: int, ps: str, rt: str, pty: int = 10) -> list[list[int]]:
    """One cycle of groups: four 0A groups for the 8-char PS and sixteen 2A
    groups for the 64-char RadioText (layout per applyGroup, rds.go:477-502)."""
    ps = (ps + " " * 8)[:8]
    rt = (rt + " " * 64)[:64]
    groups = []
    for addr in range(4):
        b = (0 << 12) | (0 << 11) | (1 << 10) | ((pty & 0x1F) << 5) | addr
        c = 0xE0CD  # alternative-frequency filler
        d = (ord(ps[2 * addr]) << 8) | ord(ps[2 * addr + 1])
        groups.append([rds_block(pi, OFF_A), rds_block(b, OFF_B), rds_block(c, OFF_C), rds_block(d, OFF_D)])
    for addr in range(16):
        b = (2 << 12) | (0 << 11) | (1 << 10) | ((pty & 0x1F) << 5) | addr
        c = (ord(rt[4 * addr]) << 8) | ord(rt[4 * addr + 1])
        d = (ord(rt[4 * addr + 2]) << 8) | ord(rt[4 * addr + 3])
        groups.append([rds_block(pi, OFF_A), rds_block(b, OFF_B), rds_block(c, OFF_C), rds_block(d, OFF_D)])
    return groups


def rds_bits(groups: list[list[int]], n_bits: int) -> np.ndarray:
    """Data bits (MSB first per block), cycling through the groups."""
    seq = []
    for g in groups:
        for blk in g:
            for i in range(25, -1, -1):
                seq.append((blk >> i) & 1)
    seq = np.array(seq, dtype=np.uint8)
    reps = n_bits // seq.size + 1
    return np.tile(seq, reps)[:n_bits]


def rds_symbols(bits: np.ndarray) -> np.ndarray:
    """Differential encoding (e[i] = e[i-1] xor b[i]) and +-1 BPSK levels."""
    e = np.bitwise_xor.accumulate(bits.astype(np.uint8))
    return (2.0 * e.astype(np.float64) - 1.0)


def random_station_text(rng: np.random.Generator):
    letters = np.array(list("ABCDEFGHIJKLMNOPQRSTUVWXYZ0123456789"))
    pi = int(rng.integers(0x1000, 0xFFFF))
    ps = "".join(rng.choice(letters, 8))
    words = ["".join(rng.choice(letters, int(rng.integers(3, 9)))) for _ in range(10)]
    rt = (" ".join(words))[:64]
    return pi, ps, rt


# --------------------------------------------------------------------------
# station models
# --------------------------------------------------------------------------

@dataclass
class WFMStation:
    offset_hz: float
    amplitude: float
    tones_l: list  # (freq, amp, phase)
    tones_r: list
    pi: int
    ps: str
    rt: str
    symbols: np.ndarray  # +-1 RDS levels
    deviation_hz: float = 75000.0
    pilot: float = 0.10
    rds: float = 0.05
    rds_phase: float = 0.0
    phase0: float = 0.0


def make_wfm_station(rng: np.random.Generator, offset_hz: float, amplitude: float, seconds: float,
                     n_tones: int = 4) -> WFMStation:
    def tones():
        # program-like spectrum: tones anywhere in 100 Hz - 15 kHz, level
        # falling with frequency as broadcast audio does
        f = rng.uniform(100.0, 15000.0, n_tones)
        a = (0.8 / n_tones) * rng.uniform(0.5, 1.0, n_tones) / (1.0 + f / 1500.0) ** 2
        ph = rng.uniform(0, 2 * math.pi, n_tones)
        return [(float(f[i]), float(a[i]), float(ph[i])) for i in range(n_tones)]

    pi, ps, rt = random_station_text(rng)
    n_bits = int(seconds * RDS_BAUD) + 64
    sym = rds_symbols(rds_bits(rds_groups(pi, ps, rt), n_bits))
    return WFMStation(offset_hz, amplitude, tones(), tones(), pi, ps, rt, sym,
                      rds_phase=float(rng.uniform(0, 2 * math.pi)), phase0=float(rng.uniform(0, 2 * math.pi)))


@dataclass
class NarrowStation:
    """NFM / AM / USB / LSB / CW channel."""
    kind: str
    offset_hz: float
    amplitude: float
    tones: list
    deviation_hz: float = 2500.0
    mod_index: float = 0.6
    wpm: float = 20.0
    key_seed: int = 0
    phase0: float = 0.0


def make_narrow_station(rng, kind: str, offset_hz: float, amplitude: float) -> NarrowStation:
    f = rng.uniform(300.0, 2700.0, 3)
    a = rng.uniform(0.3, 1.0, 3)
    a = a / a.sum()
    ph = rng.uniform(0, 2 * math.pi, 3)
    tones = [(float(f[i]), float(a[i]), float(ph[i])) for i in range(3)]
    return NarrowStation(kind, offset_hz, amplitude, tones, mod_index=float(rng.uniform(0.3, 0.9)),
                         wpm=float(rng.uniform(10, 30)), key_seed=int(rng.integers(1 << 30)),
                         phase0=float(rng.uniform(0, 2 * math.pi)))


class WidebandScene:
    """Block generator: sum of stations plus AWGN, cf32 blocks of `block`
    samples, phase-continuous across blocks."""

    def __init__(self, sample_rate: int, block: int, stations: list, noise_sigma: float, seed: int,
                 device="cpu"):
        self.fs = sample_rate
        self.block = block
        self.stations = stations
        self.noise_sigma = noise_sigma
        self.seed = seed
        self.device = torch.device(device)
        self._fm_phase = [st.phase0 for st in stations]
        self._t0 = 0  # absolute sample index of the next block
        self._gen = torch.Generator(device=self.device)
        self._gen.manual_seed(seed)

    def _tone_sum(self, tones, t):
        out = torch.zeros_like(t)
        for f, a, ph in tones:
            out += a * torch.sin(2 * math.pi * f * t + ph)
        return out

    def _wfm_mpx(self, st: WFMStation, t):
        left = self._tone_sum(st.tones_l, t)
        right = self._tone_sum(st.tones_r, t)
        lpr = 0.5 * (left + right)
        lmr = 0.5 * (left - right)
        w = 2 * math.pi * PILOT_HZ
        mpx = lpr + lmr * torch.sin(2 * w * t) + st.pilot * torch.sin(w * t)
        # RDS: cosine-interpolated +-1 symbol levels on a 57 kHz carrier
        sym = torch.as_tensor(st.symbols, dtype=torch.float64, device=self.device)
        pos = t * RDS_BAUD
        k = torch.floor(pos).long().clamp_(0, sym.numel() - 2)
        frac = pos - torch.floor(pos)
        c = 0.5 * (1 + torch.cos(math.pi * frac))
        level = sym[k] * c + sym[k + 1] * (1 - c)
        mpx = mpx + st.rds * level * torch.cos(3 * w * t + st.rds_phase)
        return mpx

    def _narrow(self, st: NarrowStation, t, idx):
        fs = self.fs
        msg = self._tone_sum(st.tones, t)
        if st.kind == "NFM":
            ph = torch.cumsum(2 * math.pi * st.deviation_hz / fs * msg, 0)
            return torch.exp(1j * ph.to(torch.float64)), ph
        if st.kind == "AM":
            env = 1.0 + st.mod_index * msg
            return env.to(torch.complex128), None
        if st.kind in ("USB", "LSB"):
            # analytic single-sideband: sum of tones rotated up (USB) or down (LSB)
            sgn = 1.0 if st.kind == "USB" else -1.0
            z = torch.zeros_like(t, dtype=torch.complex128)
            for f, a, phs in st.tones:
                z += a * torch.exp(1j * (sgn * 2 * math.pi * f * t + phs))
            return z, None
        # CW: on/off keyed carrier with 5 ms raised-cosine edges
        dot = 1.2 / st.wpm
        g = np.random.default_rng(st.key_seed)
        n_el = int(t[-1].item() / dot) + 4 if t.numel() else 4
        keys = torch.as_tensor(g.integers(0, 2, n_el + 2).astype(np.float64), device=self.device)
        pos = t / dot
        k = torch.floor(pos).long().clamp_(0, n_el)
        frac = pos - torch.floor(pos)
        edge = torch.clamp(frac * dot / 0.005, max=1.0)
        env = keys[k] * (0.5 - 0.5 * torch.cos(math.pi * edge)) + keys[k] * 0  # keyed level
        env = torch.where(keys[k] > 0, env, torch.zeros_like(env))
        return env.to(torch.complex128), None

    def next_block(self) -> torch.Tensor:
        n = self.block
        fs = self.fs
        idx = torch.arange(self._t0, self._t0 + n, dtype=torch.float64, device=self.device)
        t = idx / fs
        acc = torch.zeros(n, dtype=torch.complex128, device=self.device)
        for si, st in enumerate(self.stations):
            if isinstance(st, WFMStation):
                mpx = self._wfm_mpx(st, t)
                inst = 2 * math.pi * st.deviation_hz / fs * mpx
                ph = self._fm_phase[si] + torch.cumsum(inst, 0)
                self._fm_phase[si] = float(ph[-1].item()) % (2 * math.pi)
                base = st.amplitude * torch.exp(1j * ph)
            else:
                base, ph = self._narrow(st, t, idx)
                if ph is not None:
                    base = st.amplitude * torch.exp(1j * (self._fm_phase[si] + ph))
                    self._fm_phase[si] = float((self._fm_phase[si] + ph[-1]).item()) % (2 * math.pi)
                else:
                    base = st.amplitude * base * complex(math.cos(st.phase0), math.sin(st.phase0))
            rot = torch.exp(1j * ((2 * math.pi * st.offset_hz / fs) * (idx % fs)))
            acc += base * rot
        if self.noise_sigma > 0:
            nz = torch.randn(2, n, generator=self._gen, dtype=torch.float32, device=self.device)
            acc += (self.noise_sigma / math.sqrt(2)) * torch.complex(nz[0], nz[1]).to(torch.complex128)
        self._t0 += n
        return acc.to(torch.complex64)


def noise_sigma_for_snr(amplitude: float, snr_db: float, bw_hz: float, fs: float) -> float:
    """Complex noise std over the full band such that a station of this
    amplitude has `snr_db` in `bw_hz`."""
    n0 = amplitude ** 2 / (10 ** (snr_db / 10)) / bw_hz  # noise power per Hz
    return math.sqrt(n0 * fs)


# --------------------------------------------------------------------------
# benchmark-configuration scenes
# --------------------------------------------------------------------------

CONFIG_SEEDS = {0: 0x5EED0000, 1: 0x5EED0001, 2: 0x5EED0002, 3: 0x5EED0003, 4: 0x5EED0004}


def plain_wfm_scene(device="cpu", block=262144, seed=CONFIG_SEEDS[0]):
    """Plain case: 2.4 MS/s, one WFM station at +300 kHz, 30 dB SNR."""
    rng = np.random.default_rng(seed)
    fs = 2_400_000
    st = make_wfm_station(rng, 300_000.0, 1.0, seconds=20 * block / fs + 1)
    sigma = noise_sigma_for_snr(1.0, 30.0, 200_000.0, fs)
    return WidebandScene(fs, block, [st], sigma, seed, device), [st]


def fm_band_scene(device="cpu", block=1 << 20, n_stations=40, seconds=8.0, seed=CONFIG_SEEDS[1]):
    """FM band batch: 10 MS/s, 40 stations on a 200 kHz grid, 10-40 dB SNR."""
    rng = np.random.default_rng(seed)
    fs = 10_000_000
    offsets = [(-(n_stations // 2) + i) * 200_000.0 + 100_000.0 for i in range(n_stations)]
    snrs = rng.uniform(10.0, 40.0, n_stations)
    noise_amp = 1.0
    stations = []
    for i, off in enumerate(offsets):
        # noise reference: unit-amplitude station at 0 dB would have snr 0
        amp = math.sqrt(10 ** (snrs[i] / 10)) * 0.01
        stations.append(make_wfm_station(rng, off, amp, seconds=seconds))
    sigma = noise_sigma_for_snr(0.01 * noise_amp, 0.0, 200_000.0, fs)
    return WidebandScene(fs, block, stations, sigma, seed, device), stations


# Channel parameters per mode, as the benchmark configurations give them:
# (mode name, output rate, FIR taps, extraction bandwidth).  WFM channels are
# stereo with RDS (FM band batch); the narrow modes follow the mixed batch.
MODE_TABLE = {
    "WFM": (312_500, 256, 250_000.0),
    "NFM": (25_000, 512, 12_500.0),
    "AM": (25_000, 384, 10_000.0),
    "USB": (12_500, 256, 3_000.0),
    "LSB": (12_500, 256, 3_000.0),
    "CW": (5_000, 128, 500.0),
}


def mixed_scene(device="cpu", block=1 << 20, seed=CONFIG_SEEDS[2]):
    """Mixed-mode uneven batch: 10 MS/s, 120 channels at random non-overlapping
    offsets (25 kHz grid) with SNR 5-35 dB: 40 NFM, 30 AM, 15 USB, 15 LSB,
    20 CW.  Returns the scene and [(kind, offset_hz)] per channel."""
    rng = np.random.default_rng(seed)
    fs = 10_000_000
    kinds = ["NFM"] * 40 + ["AM"] * 30 + ["USB"] * 15 + ["LSB"] * 15 + ["CW"] * 20
    grid = np.arange(-4_900_000.0, 4_900_001.0, 25_000.0)
    offs = rng.choice(grid, size=len(kinds), replace=False)
    snrs = rng.uniform(5.0, 35.0, len(kinds))
    stations, chans = [], []
    for kind, off, snr in zip(kinds, offs, snrs):
        bw = MODE_TABLE[kind][2]
        amp = math.sqrt(10 ** (snr / 10)) * 0.01 * math.sqrt(bw / 12_500.0)
        stations.append(make_narrow_station(rng, kind, float(off), amp))
        chans.append((kind, float(off)))
    sigma = noise_sigma_for_snr(0.01, 0.0, 12_500.0, fs)
    return WidebandScene(fs, block, stations, sigma, seed, device), chans


def serving_scene(device="cpu", block=262144, seconds=10.0, seed=CONFIG_SEEDS[3]):
    """Serving stream source: a continuous 10 MS/s band with 12 WFM stations
    (stereo + RDS) and 48 narrow stations (NFM / AM / SSB / CW) at random
    non-overlapping positions, SNR 5-35 dB, plus AWGN.  Demod requests land
    at uniform-random frequencies over the band, on a station or on noise."""
    rng = np.random.default_rng(seed)
    fs = 10_000_000
    wfm_grid = np.arange(-4_700_000.0, 4_700_001.0, 400_000.0)
    wfm_offs = rng.choice(wfm_grid, size=12, replace=False)
    narrow_grid = np.array([f for f in np.arange(-4_900_000.0, 4_900_001.0, 25_000.0)
                            if np.min(np.abs(wfm_offs - f)) > 150_000.0])
    narrow_offs = rng.choice(narrow_grid, size=48, replace=False)
    kinds = ["NFM"] * 16 + ["AM"] * 12 + ["USB"] * 6 + ["LSB"] * 6 + ["CW"] * 8
    stations = []
    for off in wfm_offs:
        amp = math.sqrt(10 ** (rng.uniform(5.0, 35.0) / 10)) * 0.01
        stations.append(make_wfm_station(rng, float(off), amp, seconds=seconds + 1))
    for kind, off in zip(kinds, narrow_offs):
        bw = MODE_TABLE[kind][2]
        amp = math.sqrt(10 ** (rng.uniform(5.0, 35.0) / 10)) * 0.01 * math.sqrt(bw / 12_500.0)
        stations.append(make_narrow_station(rng, kind, float(off), amp))
    sigma = noise_sigma_for_snr(0.01, 0.0, 200_000.0, fs)
    return WidebandScene(fs, block, stations, sigma, seed, device), stations


HEADROOM_FS = 61_440_000


def headroom_scene(device="cpu", block=1 << 20, seconds=4.0, seed=CONFIG_SEEDS[4]):
    """Headroom stress source: a continuous 61.44 MS/s band with 48 WFM
    stations (stereo + RDS) on a 400 kHz grid and 160 narrow stations (NFM /
    AM / SSB / CW) at random non-overlapping positions, SNR 5-35 dB, plus
    AWGN.  Returns the scene, the WFM offsets and the narrow stations."""
    rng = np.random.default_rng(seed)
    fs = HEADROOM_FS
    wfm_grid = np.arange(-30_000_000.0, 30_000_001.0, 400_000.0)
    wfm_offs = np.sort(rng.choice(wfm_grid, size=48, replace=False))
    narrow_grid = np.array([f for f in np.arange(-30_400_000.0, 30_400_001.0, 25_000.0)
                            if np.min(np.abs(wfm_offs - f)) > 150_000.0])
    narrow_offs = rng.choice(narrow_grid, size=160, replace=False)
    kinds = ["NFM"] * 54 + ["AM"] * 40 + ["USB"] * 20 + ["LSB"] * 20 + ["CW"] * 26
    stations = []
    for off in wfm_offs:
        amp = math.sqrt(10 ** (rng.uniform(5.0, 35.0) / 10)) * 0.01
        stations.append(make_wfm_station(rng, float(off), amp, seconds=seconds + 1))
    narrow = []
    for kind, off in zip(kinds, narrow_offs):
        bw = MODE_TABLE[kind][2]
        amp = math.sqrt(10 ** (rng.uniform(5.0, 35.0) / 10)) * 0.01 * math.sqrt(bw / 12_500.0)
        st = make_narrow_station(rng, kind, float(off), amp)
        stations.append(st)
        narrow.append(st)
    sigma = noise_sigma_for_snr(0.01, 0.0, 200_000.0, fs)
    return WidebandScene(fs, block, stations, sigma, seed, device), [float(o) for o in wfm_offs], narrow

