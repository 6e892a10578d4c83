"""Long-window stereo pilot detector on the GPU (gpud_pilot_*) against the
oracle restatement of classifier.StereoPilotPresent / estimateWFMPilot:
identical decisions and best bins, the max / median ratio within 1e-6."""
import numpy as np
import pytest

import gpudemod as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _mpx_baseband(fs, seconds, pilot, snr_db, seed, pilot_hz=19000.0):
    """FM carrier at DC modulated (75 kHz deviation) by program tones plus a
    pilot at `pilot` of full deviation, complex AWGN."""
    rng = np.random.default_rng(seed)
    n = int(fs * seconds)
    t = np.arange(n) / fs
    prog = 0.3 * np.sin(2 * np.pi * rng.uniform(300, 3000) * t) + 0.2 * np.sin(2 * np.pi * rng.uniform(3e3, 12e3) * t)
    mpx = prog + pilot * np.sin(2 * np.pi * pilot_hz * t)
    ph = np.cumsum(2 * np.pi * 75000 * mpx / fs)
    sigma = 10 ** (-snr_db / 20)
    x = np.exp(1j * ph) + sigma * (rng.standard_normal(n) + 1j * rng.standard_normal(n)) / np.sqrt(2)
    return x.astype(np.complex64)


CASES = [  # (fs, seconds, pilot level, snr dB, pilot offset Hz)
    (312_500, 0.6, 0.10, 30, 0), (312_500, 0.6, 0.0, 30, 0), (300_000, 0.7, 0.01, 10, 37),
    (192_000, 2.0, 0.10, 40, -260), (250_000, 0.5, 0.002, 5, 0), (312_501, 0.6, 0.10, 20, 0),
    (312_500, 0.05, 0.10, 30, 0), (20_000, 0.5, 0.1, 30, 0), (312_500, 0.6, 0.004, 0, 500),
]


@pytest.mark.parametrize("window", [True, False])
def test_pilot_batch_matches_oracle(cuda, window):
    xs = [_mpx_baseband(fs, sec, p, snr, 100 + i, 19000.0 + off) for i, (fs, sec, p, snr, off) in enumerate(CASES)]
    rates = [c[0] for c in CASES]
    det = G.StereoPilotDetector(max_jobs=16, max_samples=1 << 19)
    try:
        got = det.run(xs, rates, window=window)
    finally:
        det.close()
    presents = []
    for (fs, *_), x, g in zip(CASES, xs, got):
        lk, ratio, best, med, _ = O.stereo_pilot(x, fs, window=window)
        assert g["present"] == lk, (fs, g, ratio)
        presents.append(lk)
        if fs >= 40_000:
            assert g["best_hz"] == best, (fs, g["best_hz"], best)
            assert abs(g["ratio"] - ratio) <= 1e-6 * max(1.0, ratio), (fs, g["ratio"], ratio)
            assert abs(g["median"] - med) <= 1e-6 * med
        else:
            assert not g["present"]
    assert any(presents) and not all(presents)
