"""Job construction (cmd/sdrd): the package's rules against the oracle's C
restatement, exactly, over common SDR sample rates and every mode; plus the
reference's own snapOutRate test (cmd/sdrd/snap_test.go:5-26)."""
import numpy as np
import pytest

from gpudemod import jobs as J
from oracle import oracle as O

SAMPLE_RATES = [1_920_000, 2_000_000, 2_048_000, 2_400_000, 2_500_000, 3_200_000, 4_000_000, 4_096_000,
                6_000_000, 8_000_000, 10_000_000, 12_288_000, 20_000_000, 30_720_000, 61_440_000]
TARGETS = [5_000, 12_500, 25_000, 48_000, 128_000, 192_000, 200_000, 250_000, 300_000, 312_500, 500_000, 512_000]


def test_snap_out_rate_reference_cases():
    # snap_test.go:6-12, with its two properties: an exact divisor within 30 % of the target
    for sr, target in [(4096000, 200000), (4096000, 512000), (2000000, 200000), (2048000, 200000),
                       (4000000, 200000)]:
        got = J.snap_out_rate(sr, target)
        assert got > 0 and sr % got == 0
        assert 0.7 <= got / target <= 1.4
    assert J.snap_out_rate(4096000, 200000) == 204800   # the live NFM case: 20.48 snaps to 20
    assert J.snap_out_rate(4096000, 512000) == 512000   # live WFM: exact 8


@pytest.mark.parametrize("sr", SAMPLE_RATES)
def test_rates_match_oracle(sr):
    for t in TARGETS:
        assert J.snap_out_rate(sr, t) == O.snap_out_rate(sr, t), (sr, t)
        for lo in (0, 128_000, 250_000):
            assert J.nearest_exact_decimation_rate(sr, t, lo) == O.nearest_exact_decimation_rate(sr, t, lo), \
                (sr, t, lo)
    assert J.rds_extract_job(sr, 0.0).OutRate == O.rds_job_out_rate(sr)
    for mode, wfm in (("WFM", True), ("WFM_STEREO", True), ("NFM", False), ("AM", False), ("USB", False),
                      ("LSB", False), ("CW", False)):
        for snip in (sr, 128_000, 200_000, 204_800, 250_000, 256_000, 500_000, 512_000, 1_000_000):
            assert J.snippet_decim(snip, mode) == O.snippet_decim(snip, J.DEMOD_RATE[mode], wfm), (snip, mode)


def test_nearest_exact_rate_edges():
    # exact target kept; the non-divisor guard skips sr / d that does not divide sr
    assert J.nearest_exact_decimation_rate(10_000_000, 200_000, 128_000) == 200_000
    assert J.nearest_exact_decimation_rate(4_096_000, 200_000, 128_000) == 204_800
    assert J.nearest_exact_decimation_rate(2_400_000, 512_000, 128_000) == 480_000
    # nothing qualifies: the target comes back (ExactIntegerDecimation then fails)
    assert J.nearest_exact_decimation_rate(1_000_003, 200_000, 128_000) == 200_000
    assert J.nearest_exact_decimation_rate(0, 200_000, 1) == 200_000


def _signals(rng, tuner_hz, n=40):
    kinds = ["", "WFM", "WFM_STEREO", "NFM", "AM", "USB"]
    sigs = []
    for i in range(n):
        # half in the broadcast band (WFM by frequency), half outside
        f = tuner_hz + rng.uniform(-1.5e6, 1.5e6)
        sigs.append(J.Signal(i + 1, float(f), float(rng.choice([3e3, 12.5e3, 18e3, 150e3, 200e3, 300e3])),
                             str(rng.choice(kinds))))
    return sigs


@pytest.mark.parametrize("sr", [2_048_000, 2_400_000, 4_096_000, 8_000_000])
@pytest.mark.parametrize("tuner_hz", [98.0e6, 145.0e6])
@pytest.mark.parametrize("cfg", [J.ExtractionConfig(), J.ExtractionConfig(101, 1.35), J.ExtractionConfig(257, 1.2)])
def test_streaming_jobs_match_oracle(sr, tuner_hz, cfg):
    sigs = _signals(np.random.default_rng(sr + int(tuner_hz)), tuner_hz)
    want = [O.streaming_job(sr, tuner_hz, s.CenterHz, s.BWHz, s.ModType in ("WFM", "WFM_STEREO"), cfg.firTaps,
                            cfg.bwMult) for s in sigs]
    if any(w is None for w in want):
        with pytest.raises(ValueError):
            J.build_streaming_jobs(sr, tuner_hz, sigs, cfg)
        return
    got = J.build_streaming_jobs(sr, tuner_hz, sigs, cfg)
    for g, w, s in zip(got, want, sigs):
        assert (g.OffsetHz, g.Bandwidth, g.OutRate, g.NumTaps) == w
        assert g.SignalID == s.ID
        assert g.ConfigHash == O.streaming_config_hash(s.ID, g.OutRate, g.NumTaps, sr)


def test_streaming_jobs_reject_inexact_wfm_rate():
    # 512 kS/s does not divide 10 MS/s: the reference fails the batch
    sig = J.Signal(1, 98.3e6, 200e3, "")
    with pytest.raises(ValueError):
        J.build_streaming_jobs(10_000_000, 98.0e6, [sig])
    assert O.streaming_job(10_000_000, 98.0e6, 98.3e6, 200e3, False) is None


@pytest.mark.parametrize("sr", SAMPLE_RATES)
def test_batch_jobs_match_oracle(sr):
    tuner = 100.0e6
    sigs = _signals(np.random.default_rng(sr), tuner, 24)
    for g, s in zip(J.batch_extract_jobs(sr, tuner, sigs), sigs):
        w = O.batch_extract_job(sr, tuner, s.CenterHz, s.BWHz, s.ModType in ("WFM", "WFM_STEREO"))
        assert (g.OffsetHz, g.BW, g.OutRate) == w


def test_production_channel_classes():
    # 4.096 MS/s (the reference's live SDR rate): WFM extracted at 512 kS/s then
    # decimated by 2 to 256 kS/s; narrow signals at 204.8 kS/s then by 4 to 51.2 kS/s
    sigs = [J.Signal(1, 145.3e6, 180e3, "WFM"), J.Signal(2, 144.0e6, 12.5e3, "NFM")]
    jw, jn = J.build_streaming_jobs(4_096_000, 145.0e6, sigs, J.ExtractionConfig(101, 1.35))
    cw = J.production_channel(jw, "WFM_STEREO", rds=True)
    cn = J.production_channel(jn, "NFM")
    assert (cw["out_rate"], cw["demod_decim"], cw["num_taps"], cw["bandwidth"]) == (512_000, 2, 101, 250_000.0)
    assert (cn["out_rate"], cn["demod_decim"], cn["bandwidth"]) == (204_800, 4, 20_000.0)
