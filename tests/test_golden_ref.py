"""The CPU oracle pinned to the reference's own code without a GPU:
tests/golden/ref_launchers.npz holds outputs of the reference's GPU launchers
(its native/exports.cu, compiled from the reference tree into oracle/_ref and
run once by tests/golden/make_ref_golden.py) on deterministic inputs.  The
oracle's streaming polyphase extraction (streaming_host_core.go:5-64
restated) must reproduce the reference kernel chunk by chunk -- outputs,
carried history length, phase count and NCO phase -- and its discriminator
the reference's `gpud_launch_fm_discrim_cuda`, and its legacy batch slot the
reference's launchers composed as the Windows batch runner composes them,
within the float32 roundings that separate a GPU kernel from a CPU
restatement."""
import hashlib
import math
import os

import numpy as np
import pytest

from oracle import oracle as O
from signals import make_deterministic_iq, make_tone_noise_iq, max_abs, rel_l2

FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_launchers.npz")


@pytest.fixture(scope="module")
def golden():
    return dict(np.load(FIX))


def _sha(x):
    return np.frombuffer(hashlib.sha256(np.ascontiguousarray(x).tobytes()).digest(), np.uint8)


@pytest.mark.parametrize("case", [0, 1, 2])
def test_oracle_streaming_extraction_matches_reference_kernel(golden, case):
    fs = int(golden["fs"])
    chunks = [int(c) for c in golden["chunks"]]
    x = make_tone_noise_iq(sum(chunks), 0.021)
    assert np.array_equal(_sha(x), golden["stateful_in_sha256"])  # the input the reference saw
    taps, decim, offset = golden[f"stateful{case}_geom"]
    taps, decim = int(taps), int(decim)
    poly = O.build_polyphase_taps_phase_major(O.base_taps_f32(20_000, fs, taps), decim)
    assert np.array_equal(poly, golden[f"stateful{case}_poly"])
    hist, phase, pc, pos = np.zeros(0, np.complex64), 0.0, 0, 0
    for j, n in enumerate(chunks):
        chunk = x[pos:pos + n]
        pos += n
        got, phase, pc, hist = O.run_host_core(chunk, fs, float(offset), phase, pc, taps, decim, hist, poly)
        want = golden[f"stateful{case}_out{j}"]
        hl, rpc, rph = golden[f"stateful{case}_state{j}"]
        assert got.size == want.size, (j, got.size, want.size)
        if want.size:
            assert max_abs(got, want) <= 1e-5, (j, max_abs(got, want))
        assert hist.size == int(hl) and pc == int(rpc), j
        assert abs(math.remainder(phase - float(rph), 2 * math.pi)) <= 1e-9, j


@pytest.mark.parametrize("case", [0, 1])
def test_oracle_discriminator_matches_reference_kernel(golden, case):
    x = (make_tone_noise_iq(20_000, 0.3), make_deterministic_iq(20_000))[case]
    assert np.array_equal(_sha(x), golden[f"discrim{case}_in_sha256"])
    want = golden[f"discrim{case}_out"]
    got = O.fm_discrim(x)
    assert got.size == want.size
    # the oracle takes the products and atan2 in float64 (the reference's CPU
    # path); the reference kernel in float32
    assert max_abs(got, want) <= 2e-6 and rel_l2(got, want) <= 1e-6


def test_pin_detects_a_planted_offset_error(golden):
    """Negative control: the oracle run 1 Hz off the reference's offset leaves
    the bound after a few thousand samples (the pin has teeth)."""
    fs = int(golden["fs"])
    chunks = [int(c) for c in golden["chunks"]]
    x = make_tone_noise_iq(sum(chunks), 0.021)
    taps, decim, offset = golden["stateful0_geom"]
    taps, decim = int(taps), int(decim)
    poly = golden["stateful0_poly"]
    hist, phase, pc, pos, worst = np.zeros(0, np.complex64), 0.0, 0, 0, 0.0
    for j, n in enumerate(chunks):
        got, phase, pc, hist = O.run_host_core(x[pos:pos + n], fs, float(offset) + 1.0, phase, pc, taps, decim,
                                               hist, poly)
        pos += n
        want = golden[f"stateful0_out{j}"]
        if want.size:
            worst = max(worst, max_abs(got, want))
    assert worst > 1e-3, worst


@pytest.mark.parametrize("geom", [0, 1])
def test_oracle_batch_slot_matches_reference_chain(golden, geom):
    """The legacy batch slot (frequency shift from the job's start phase, FIR
    v2, decimation) as the reference's own launchers compose it, against the
    oracle's restatement of batch_runner_windows.go:142-182."""
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    import make_ref_golden as M
    fs, jobs = M.SLOTS[geom]
    x = M.slot_input(fs, jobs)
    assert np.array_equal(_sha(x), golden[f"slot{geom}_in_sha256"])
    for j, (off, bw, rate, p0) in enumerate(jobs):
        want = golden[f"slot{geom}_job{j}_out"]
        got, grate, _ = O.batch_slot(x, fs, off, bw, rate, p0)
        assert grate == rate and got.size == want.size, (j, got.size, want.size)
        assert rel_l2(got, want) <= 1e-6, (j, rel_l2(got, want))
