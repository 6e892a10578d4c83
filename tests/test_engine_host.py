"""Host-side pieces of the Engine mirror: the tap design the library exports
(dsp.LowpassFIR, dsp/fir.go:6-28) equals the oracle's restatement bit for
bit, and Go's math.Round (half away from zero) as the decimation rule uses it."""
import numpy as np

import gpudemod as G
from oracle import oracle as O


def test_lowpass_fir_matches_oracle_exactly():
    for cutoff, fs, taps in [(125_000.0, 2_400_000, 101), (6_250.0, 10_000_000, 101), (200.0, 48_000, 64),
                             (90_000.0, 512_000, 101), (0.0, 2_400_000, 33), (-5.0, 1_000, 7)]:
        got = G.LowpassFIR(cutoff, fs, taps)
        want = O.lowpass_fir(cutoff, fs, taps)
        assert got.size == (taps | 1) and np.array_equal(got, want)


def test_go_round():
    assert [G._go_round(x) for x in (0.0, 0.49999999999999994, 0.5, 1.5, 2.5, 208.33, 52.08)] == \
        [0, 0, 1, 2, 3, 208, 52]
