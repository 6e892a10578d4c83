"""SDRIQ001 snapshots (gpud_iqfile_*, internal/iqfile/iqfile.go): the
reference's round-trip and looping-replay tests, the format's header bytes,
and the errors for a bad magic or a truncated file -- host paths only."""
import struct

import numpy as np
import pytest

import gpudemod as G
from gpudemod import iqfile


def test_round_trip(tmp_path):
    """iqfile_test.go:9-29."""
    iq = (np.arange(1000) * 0.001 - 1j * np.arange(1000) * 0.002).astype(np.complex64)
    p = tmp_path / "snap.cf32"
    iqfile.write(p, iq, 4_096_000, 101.5e6)
    got, meta = iqfile.read(p)
    assert (meta.SampleRate, meta.CenterHz, meta.Samples) == (4_096_000, 101.5e6, 1000)
    assert np.array_equal(got, iq)
    raw = p.read_bytes()
    assert raw[:8] == b"SDRIQ001" and len(raw) == 32 + 8 * 1000
    assert struct.unpack("<qdq", raw[8:32]) == (4_096_000, 101.5e6, 1000)
    assert np.array_equal(np.frombuffer(raw[32:], np.complex64), iq)


def test_replay_source_loops(tmp_path):
    """iqfile_test.go:31-51: three samples read as seven."""
    p = tmp_path / "s.cf32"
    iqfile.write(p, np.array([1, 2, 3], np.complex64), 1000, 0.0)
    s = iqfile.Source(p)
    assert np.array_equal(s.read_iq(7), np.array([1, 2, 3, 1, 2, 3, 1], np.complex64))
    assert np.array_equal(s.read_iq(2), np.array([2, 3], np.complex64))
    s.close()


def test_errors_and_empty(tmp_path):
    p = tmp_path / "bad.cf32"
    p.write_bytes(b"NOTIQ001" + bytes(24))
    with pytest.raises(G.GPUDError) as e:
        iqfile.read(p)
    assert e.value.code == -34
    q = tmp_path / "short.cf32"
    iqfile.write(q, np.ones(10, np.complex64), 1000, 0.0)
    q.write_bytes(q.read_bytes()[:-8])  # header says 10, file holds 9
    with pytest.raises(G.GPUDError):
        iqfile.read(q)
    with pytest.raises(G.GPUDError) as e:
        iqfile.read(tmp_path / "missing.cf32")
    assert e.value.code == -33
    z = tmp_path / "empty.cf32"
    iqfile.write(z, np.zeros(0, np.complex64), 48000, 1e6)
    s = iqfile.Source(z, paced=False)
    assert np.array_equal(s.read_iq(4), np.zeros(4, np.complex64))
    assert s.buffer_samples() == 0
