"""Streaming extraction on the GPU (libgpudemod_kernels.so through its C ABI)
against the CPU oracle -- restates gpudemod/streaming_gpu_exec_test.go:33-121
and extends it to the benchmark geometries (even tap counts, uneven batches)."""
import math

import numpy as np
import pytest

import gpudemod as G
from oracle import oracle as O
from signals import chunks_of, make_deterministic_iq, make_tone_noise_iq, max_abs, phase_diff, rel_l2

pytestmark = pytest.mark.gpu

JOB = G.StreamingExtractJob(SignalID=1, OffsetHz=12500, Bandwidth=20000, OutRate=200000, NumTaps=65, ConfigHash=777)


def _ojob(j):
    return O.StreamingExtractJob(j.SignalID, j.OffsetHz, j.Bandwidth, j.OutRate, j.NumTaps, j.ConfigHash)


def run_sequence_against_oracle(steps, fs=4_000_000, sample_tol=1e-5, phase_tol=1e-9):
    runner = G.NewBatchRunner(max(1, max(len(s[0]) for s in steps)), fs)
    oracle = O.CPUOracleRunner(fs)
    try:
        for idx, (iq, jobs) in enumerate(steps):
            got = runner.StreamingExtractGPU(iq, jobs)
            want = oracle.StreamingExtract(iq, [_ojob(j) for j in jobs])
            assert len(got) == len(want)
            for g, w in zip(got, want):
                assert g.SignalID == w.SignalID
                assert g.Rate == w.Rate
                assert g.NOut == w.NOut, (idx, g.NOut, w.NOut)
                assert g.PhaseCount == w.PhaseCount
                assert g.HistoryLen == w.HistoryLen
                assert max_abs(g.IQ, w.IQ) <= sample_tol, (idx, max_abs(g.IQ, w.IQ))
                assert phase_diff(g.NCOPhase, oracle.States[g.SignalID].NCOPhase) <= phase_tol
            assert set(oracle.States) == {j.SignalID for j in jobs}
    finally:
        runner.Close()


def test_exec_matches_oracle_deterministic_iq(cuda):
    iq = make_deterministic_iq(1500)
    steps = [(c, [JOB]) for c in chunks_of(iq, [0, 1, 2, 17, 63, 64, 65, 129, 511])]
    run_sequence_against_oracle(steps)


def test_exec_matches_oracle_tone_noise_iq(cuda):
    iq = make_tone_noise_iq(4096, 0.023)
    steps = [(c, [JOB]) for c in chunks_of(iq, [7, 20, 3, 63, 64, 65, 777])]
    run_sequence_against_oracle(steps)


def test_exec_lifecycle(cuda):
    a = G.StreamingExtractJob(11, 12500, 20000, 200000, 65, 1001)
    b = G.StreamingExtractJob(22, -18750, 16000, 100000, 33, 2002)
    a_reset = G.StreamingExtractJob(11, 12500, 20000, 200000, 65, 1002)
    steps = [
        (make_deterministic_iq(512), [a, b]),                      # prime both signals
        (np.zeros(0, np.complex64), [a_reset, b]),                # config reset with zero new samples
        (make_tone_noise_iq(96, 0.041), [a_reset]),               # signal b disappears
        (make_deterministic_iq(160), [a_reset, b]),               # signal b reappears fresh
        (make_tone_noise_iq(65, 0.017), [a_reset, b]),            # small history-boundary chunk
    ]
    run_sequence_against_oracle(steps)


@pytest.mark.parametrize("fs,out_rate,taps,bw,offset", [
    (2_400_000, 300_000, 128, 250_000, 300_000.0),      # plain-method geometry (D=8, L=16)
    (10_000_000, 312_500, 256, 250_000, -1_300_000.0),  # FM-band geometry (D=32, L=8)
    (10_000_000, 25_000, 512, 15_000, 2_345_678.0),     # NFM (D=400, L=2, wide path)
    (10_000_000, 12_500, 256, 3_000, -3_210_000.0),     # SSB (D=800, L=1)
    (10_000_000, 5_000, 128, 500, 777_777.0),           # CW (D=2000)
    (10_000_000, 625_000, 1024, 400_000, 123_456.0),    # D=16, L=64 (wide path)
    (10_000_000, 100_000, 1000, 60_000, -45_000.0),     # D=100, L=10
])
def test_extract_geometries_match_oracle(cuda, fs, out_rate, taps, bw, offset):
    rng = np.random.default_rng(taps)
    n_blocks, block = 3, 65_536 + 123
    x = (rng.standard_normal(n_blocks * block) + 1j * rng.standard_normal(n_blocks * block)).astype(np.complex64)
    x += make_tone_noise_iq(x.size, 2 * math.pi * offset / fs)
    job = G.StreamingExtractJob(5, offset, bw, out_rate, taps, 42)
    steps = [(x[i * block:(i + 1) * block], [job]) for i in range(n_blocks)]
    runner = G.NewBatchRunner(block, fs)
    oracle = O.CPUOracleRunner(fs)
    try:
        for iq, jobs in steps:
            g = runner.StreamingExtractGPU(iq, jobs)[0]
            w = oracle.StreamingExtract(iq, [_ojob(j) for j in jobs])[0]
            assert (g.NOut, g.PhaseCount, g.HistoryLen) == (w.NOut, w.PhaseCount, w.HistoryLen)
            assert rel_l2(g.IQ, w.IQ) <= 1e-5, rel_l2(g.IQ, w.IQ)
            assert phase_diff(g.NCOPhase, oracle.States[5].NCOPhase) <= 1e-9
    finally:
        runner.Close()


def test_uneven_batch_in_one_launch_matches_oracle(cuda):
    fs = 10_000_000
    jobs = [
        G.StreamingExtractJob(1, -3_900_000, 250_000, 312_500, 256, 1),
        G.StreamingExtractJob(2, 1_000_000, 15_000, 25_000, 512, 2),
        G.StreamingExtractJob(3, 2_000_000, 12_000, 25_000, 384, 3),
        G.StreamingExtractJob(4, -2_500_000, 3_000, 12_500, 256, 4),
        G.StreamingExtractJob(5, 3_300_000, 500, 5_000, 128, 5),
        G.StreamingExtractJob(6, 500_000, 100_000, 200_000, 101, 6),
        G.StreamingExtractJob(7, -700_000, 40_000, 80_000, 77, 7),
    ]
    rng = np.random.default_rng(7)
    block = 40_000
    runner = G.NewBatchRunner(block, fs)
    oracle = O.CPUOracleRunner(fs)
    try:
        for b in range(3):
            x = (rng.standard_normal(block) + 1j * rng.standard_normal(block)).astype(np.complex64)
            got = runner.StreamingExtractGPU(x, jobs)
            want = oracle.StreamingExtract(x, [_ojob(j) for j in jobs])
            for g, w in zip(got, want):
                assert (g.NOut, g.PhaseCount, g.HistoryLen) == (w.NOut, w.PhaseCount, w.HistoryLen)
                assert rel_l2(g.IQ, w.IQ) <= 1e-5, (g.SignalID, rel_l2(g.IQ, w.IQ))
    finally:
        runner.Close()


def test_invalid_decimation_rejected(cuda):
    runner = G.NewBatchRunner(1024, 4_000_000)
    try:
        with pytest.raises(G.GPUDError) as ei:
            runner.StreamingExtractGPU(make_deterministic_iq(100),
                                       [G.StreamingExtractJob(1, 0, 10000, 192_000, 65, 1)])
        assert ei.value.code == G.E_DECIM
    finally:
        runner.Close()
