"""Deterministic inputs restated from the reference's test helpers
(gpudemod/cpu_oracle_test.go:9-25, streaming_gpu_validation_helpers_test.go:16-27,
test_harness.go:16-42) plus relative-error helpers."""
import math

import numpy as np


def make_deterministic_iq(n: int) -> np.ndarray:
    i = np.arange(n, dtype=np.float64)
    a, b = 0.017 * i, 0.031 * i
    return (np.cos(a) + 0.2 * np.cos(b) + 1j * (np.sin(a) + 0.15 * np.sin(b))).astype(np.complex64)


def make_tone_noise_iq(n: int, phase_inc: float) -> np.ndarray:
    i = np.arange(n, dtype=np.float64)
    phase = phase_inc * i
    tone = np.cos(phase) + 1j * np.sin(phase)
    ni = 0.17 * np.cos(0.113 * i + 0.31) + 0.07 * np.sin(0.071 * i)
    nq = 0.13 * np.sin(0.097 * i + 0.11) - 0.05 * np.cos(0.043 * i)
    return (0.85 * tone + 0.15 * (ni + 1j * nq)).astype(np.complex64)


def make_tone_iq(n: int, phase_inc: float) -> np.ndarray:
    phase = phase_inc * np.arange(n, dtype=np.float64)
    return (np.cos(phase) + 1j * np.sin(phase)).astype(np.complex64)


def make_lowpass_taps(n: int) -> np.ndarray:
    return np.full(n, np.float32(1.0) / np.float32(n), dtype=np.float32)


def chunks_of(x, sizes):
    """makeStreamingValidationSteps: the listed chunk sizes then the remainder."""
    out, pos = [], 0
    for s in sizes:
        s = max(0, s)
        end = min(len(x), pos + s)
        out.append(x[pos:end])
        pos = end
    if pos < len(x):
        out.append(x[pos:])
    return out


def max_abs(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    assert a.shape == b.shape, (a.shape, b.shape)
    if a.size == 0:
        return 0.0
    return float(np.max(np.abs(a.astype(np.complex128) - b.astype(np.complex128))))


def rel_l2(got, want) -> float:
    got = np.asarray(got).astype(np.complex128)
    want = np.asarray(want).astype(np.complex128)
    assert got.shape == want.shape, (got.shape, want.shape)
    den = np.linalg.norm(want)
    num = np.linalg.norm(got - want)
    if den == 0:
        return float(num)
    return float(num / den)


def phase_diff(a: float, b: float) -> float:
    d = a - b
    while d > math.pi:
        d -= 2 * math.pi
    while d < -math.pi:
        d += 2 * math.pi
    return abs(d)
