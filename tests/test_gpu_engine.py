"""The single-signal Engine (gpudemod.go:81-489) and the legacy batch paths
(batch.go:20-50, batch_runner.go:61-98 with batch_runner_windows.go:99-182),
composed as the Go host composes them, against the oracle's restatement of
the same chains, at the plain config's geometry (2.4 MS/s, 262144-sample
blocks) and the mixed batch's (10 MS/s, 2^20-sample blocks).  Output counts
and rates exact; samples within rel-L2 1e-5."""
import numpy as np
import pytest

import gpudemod as G
from oracle import oracle as O
from signals import make_tone_noise_iq, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _c0_block():
    from gpudemod import synth
    scene, _ = synth.plain_wfm_scene(block=262_144)
    return 2_400_000, scene.next_block().numpy()


def _c2_block():
    from gpudemod import synth
    scene, _ = synth.mixed_scene(device="cuda", block=1 << 20, seed=synth.CONFIG_SEEDS[2])
    x = scene.next_block().cpu().numpy()
    # plus a strong tone far off centre, so the shift's phase runs through many binades
    return 10_000_000, (x + 0.3 * make_tone_noise_iq(x.size, 2.7)).astype(np.complex64)


GEOMETRIES = {
    "c0": (_c0_block, [(300_000.0, 250_000.0, 300_000), (-1_100_000.0, 12_500.0, 48_000), (0.0, 10_000.0, 200_000),
                       (700_001.5, 3_000.0, 48_000)]),
    "c2": (_c2_block, [(4_300_000.0, 12_500.0, 25_000), (-3_141_592.0, 10_000.0, 200_000),
                       (1_234_567.0, 250_000.0, 312_500), (-4_800_000.0, 3_000.0, 50_000)]),
}


@pytest.mark.parametrize("geom", ["c0", "c2"])
def test_engine_shift_filter_decimate(cuda, geom):
    make, jobs = GEOMETRIES[geom]
    fs, x = make()
    eng = G.Engine(x.size, fs)
    try:
        for off, bw, rate in jobs:
            got, grate = eng.ShiftFilterDecimate(x, off, bw, rate)
            want, wrate = O.engine_shift_filter_decimate(x, fs, off, bw, rate)
            assert grate == wrate and got.size == want.size, (off, grate, wrate, got.size, want.size)
            assert rel_l2(got, want) <= TOL, (geom, off, rel_l2(got, want))
        assert eng.LastShiftUsedGPU()
        # batch.go: per-job ShiftFilterDecimate, PhaseEnd from PhaseStart
        bj = [G.ExtractJob(off, bw, rate, 0.25 * k) for k, (off, bw, rate) in enumerate(jobs)]
        res = eng.ShiftFilterDecimateBatchWithPhase(x, bj)
        for r, j in zip(res, bj):
            want, wrate = O.engine_shift_filter_decimate(x, fs, j.OffsetHz, j.BW, j.OutRate)
            assert r.Rate == wrate and rel_l2(r.IQ, want) <= TOL
            assert r.PhaseEnd == j.PhaseStart + (-2.0 * np.pi * j.OffsetHz / fs) * x.size
        with pytest.raises(ValueError):
            eng.ShiftFilterDecimate(x, 0.0, 1e4, 0)
        assert eng.ShiftFilterDecimate(x[:0], 0.0, 1e4, 48_000) == (None, 0)
    finally:
        eng.Close()


@pytest.mark.parametrize("geom", ["c0", "c2"])
@pytest.mark.parametrize("mode", [G.DemodNFM, G.DemodWFM, G.DemodAM, G.DemodUSB, G.DemodLSB, G.DemodCW])
def test_engine_demod_sequence(cuda, geom, mode):
    """Three Demod calls in a row: the first call's taps stay (a later call
    with another bandwidth reuses them) and the BFO phase carries."""
    make, jobs = GEOMETRIES[geom]
    fs, x = make()
    off, bw, _ = jobs[1]
    eng = G.Engine(x.size, fs)
    ref = O.Engine(fs)
    try:
        for k, (a, b) in enumerate(((0, x.size // 2), (x.size // 2, x.size // 2 + 40_001), (0, x.size))):
            seg = x[a:b]
            got, grate = eng.Demod(seg, off, bw * (1 + k), mode)
            want, wrate = ref.demod(seg, off, bw * (1 + k), mode)
            assert grate == wrate and got.size == want.size, (k, grate, wrate, got.size, want.size)
            assert rel_l2(got, want) <= TOL, (geom, mode, k, rel_l2(got, want))
        assert eng.LastDemodUsedGPU()
        assert eng.DemodFused(x[:1000], off, bw, mode)[1] == grate
    finally:
        eng.Close()


@pytest.mark.parametrize("geom", ["c0", "c2"])
def test_batch_runner_shift_filter_decimate(cuda, geom):
    """BatchRunner.ShiftFilterDecimateBatch[WithPhase]: every job on its own
    stream from its PhaseStart, exact decimation, len(iq) // D outputs."""
    make, jobs = GEOMETRIES[geom]
    fs, x = make()
    br = G.NewBatchRunner(x.size, fs)
    try:
        bj = [G.ExtractJob(off, bw, rate, 1.5 - 0.7 * k) for k, (off, bw, rate) in enumerate(jobs)]
        outs, rates = br.ShiftFilterDecimateBatch(x, bj)
        res = br.ShiftFilterDecimateBatchWithPhase(x, bj)
        for j, o, r, e in zip(bj, outs, rates, res):
            want, wrate, pend = O.batch_slot(x, fs, j.OffsetHz, j.BW, j.OutRate, j.PhaseStart)
            assert r == wrate == e.Rate and o.size == want.size == e.IQ.size
            assert rel_l2(o, want) <= TOL, (geom, j.OffsetHz, rel_l2(o, want))
            assert np.array_equal(o, e.IQ)
            assert e.PhaseEnd == pend
        # fewer jobs reuse the slots; an inexact rate is refused like ExactIntegerDecimation
        o1, r1 = br.ShiftFilterDecimateBatch(x[: x.size // 2], bj[:1])
        want, wrate, _ = O.batch_slot(x[: x.size // 2], fs, bj[0].OffsetHz, bj[0].BW, bj[0].OutRate,
                                      bj[0].PhaseStart)
        assert r1[0] == wrate and rel_l2(o1[0], want) <= TOL
        with pytest.raises(ValueError):
            br.ShiftFilterDecimateBatch(x, [G.ExtractJob(0.0, 1e4, 7_000_001)])
        assert br.ShiftFilterDecimateBatch(x[:0], bj) == ([None] * len(bj), [0] * len(bj))
    finally:
        br.Close()
