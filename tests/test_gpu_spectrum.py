"""Surveillance spectrum on the device (gpud_spectrum_*) against the float64
DFT restatement of fftutil.Spectrum / WelchPSD (internal/fft/fft.go:19-55,
welch.go:15-66): fftshifted dB within 1e-6 dB, for the sizes and the Welch
call the surveillance loop makes (cmd/sdrd/pipeline_runtime.go:294-312)."""
import numpy as np
import pytest

import gpudemod as G
from gpudemod import synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_spectrum_and_welch_match_float64_dft(cuda):
    scene, _ = synth.fm_band_scene(block=1 << 18, n_stations=8, seconds=0.2)
    x = scene.next_block().numpy()
    sp = G.Spectrum(8192, 64)
    try:
        for n in (2048, 4096, 8192):
            for hann in (True, False):
                got = sp.single(x[:n], hann)
                want = O.spectrum(x[:n], O.hann(n) if hann else None)
                assert got.size == n and np.max(np.abs(got - want)) <= 1e-6, (n, hann)
            segs = 16
            need = n + (segs - 1) * n // 2  # the surveillance loop's Welch window
            got = sp.welch(x[-need:], n, 0.5, True)
            want = O.welch_psd(x[-need:], n, 0.5, O.hann(n))
            assert got.size == n and np.max(np.abs(got - want)) <= 1e-6, n
        # other overlaps, and fewer samples than a segment (Spectrum of the whole vector, no window)
        got = sp.welch(x[:20000], 2048, 0.75, True)
        assert np.max(np.abs(got - O.welch_psd(x[:20000], 2048, 0.75, O.hann(2048)))) <= 1e-6
        got = sp.welch(x[:1024], 2048, 0.5, True)
        assert got.size == 1024 and np.max(np.abs(got - O.welch_psd(x[:1024], 2048, 0.5, O.hann(2048)))) <= 1e-6
        with pytest.raises(G.GPUDError):
            sp.single(x[:3000])  # not a power of two
    finally:
        sp.close()
