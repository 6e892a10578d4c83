"""The allocation-free stateful extractor (callers that cannot allocate device
memory around the call: a real-time loop that must not stall on cudaMalloc /
cudaFree, a process whose device memory is committed to a fixed budget).  It
must give exactly what the existing entry point gives with caller-provided
scratch, call after call.  This file is collected last on purpose."""
import ctypes as C
import math

import numpy as np
import pytest

from gpudemod._lib import lib
from oracle import oracle as O
from signals import make_tone_noise_iq

pytestmark = pytest.mark.gpu

GPUD_NOALLOC_MAX_NEW = 262144
GPUD_NOALLOC_MAX_HISTORY = 4096
GPUD_E_SCRATCH = -32


def _dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def _zeros(n, dtype):
    import torch
    return torch.zeros(max(n, 1), dtype=dtype, device="cuda")


def test_noalloc_matches_caller_scratch_entry_point(cuda):
    import torch
    fs, taps, decim, offset = 2_400_000, 128, 8, 300_000.0
    base = O.base_taps_f32(250_000, fs, taps)
    poly = O.build_polyphase_taps_phase_major(base, decim)
    cap = taps - 1
    d_taps = _dev(poly)
    inc = -2 * math.pi * offset / fs
    x = make_tone_noise_iq(200_001, 0.021)
    # reference entry point state / buffers
    ha, hs = _zeros(cap, torch.complex64), _zeros(cap, torch.complex64)
    hl_a, pc_a, ph_a = C.c_int(0), C.c_int(0), C.c_double(0.0)
    # allocation-free entry point state / buffers
    hb = _zeros(cap, torch.complex64)
    hl_b, pc_b, ph_b = C.c_int(0), C.c_int(0), C.c_double(0.0)
    pos = 0
    for n in (131_071, 68_930):  # two calls in a row, state carried between them
        chunk = x[pos:pos + n]
        pos += n
        d_in = _dev(chunk)
        d_shift = _zeros(n, torch.complex64)
        out_a = _zeros(n // decim + 2, torch.complex64)
        out_b = _zeros(n // decim + 2, torch.complex64)
        na, nb = C.c_int(), C.c_int()
        rc = lib.gpud_launch_streaming_polyphase_stateful_cuda(
            d_in.data_ptr(), n, d_shift.data_ptr(), d_taps.data_ptr(), poly.size, decim, taps, ha.data_ptr(),
            hs.data_ptr(), cap, C.byref(hl_a), C.byref(pc_a), C.byref(ph_a), inc, out_a.data_ptr(),
            n // decim + 2, C.byref(na))
        assert rc == 0
        rc = lib.gpud_launch_streaming_polyphase_stateful_noalloc_cuda(
            d_in.data_ptr(), n, d_taps.data_ptr(), poly.size, decim, taps, hb.data_ptr(), cap, C.byref(hl_b),
            C.byref(pc_b), C.byref(ph_b), inc, out_b.data_ptr(), n // decim + 2, C.byref(nb))
        assert rc == 0
        assert lib.gpud_stream_sync(None) == 0
        assert (na.value, hl_a.value, pc_a.value) == (nb.value, hl_b.value, pc_b.value)
        assert ph_a.value == ph_b.value
        ga = out_a.cpu().numpy()[: na.value]
        gb = out_b.cpu().numpy()[: nb.value]
        assert np.max(np.abs(ga - gb)) <= 1e-5  # same kernels: identical in practice
        assert np.array_equal(ha.cpu().numpy()[: hl_a.value], hb.cpu().numpy()[: hl_b.value])


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda):
    import torch
    taps = torch.zeros(16, dtype=torch.float32, device="cuda")
    tp = C.c_void_p(taps.data_ptr())
    i, d = C.c_int(0), C.c_double(0.0)
    rc = lib.gpud_launch_streaming_polyphase_stateful_noalloc_cuda(
        None, GPUD_NOALLOC_MAX_NEW + 1, tp, 16, 2, 8, None, 7, C.byref(i), C.byref(i), C.byref(d), 0.0, None, 0,
        C.byref(i))
    assert rc == GPUD_E_SCRATCH
    rc = lib.gpud_launch_streaming_polyphase_stateful_noalloc_cuda(
        None, 0, tp, 16, 2, 8, None, GPUD_NOALLOC_MAX_HISTORY + 1, C.byref(i), C.byref(i), C.byref(d), 0.0, None,
        0, C.byref(i))
    assert rc == GPUD_E_SCRATCH
    # the base entry point's argument codes come before the scratch limits
    rc = lib.gpud_launch_streaming_polyphase_stateful_noalloc_cuda(
        None, GPUD_NOALLOC_MAX_NEW + 1, tp, 16, 2, 8, None, 7, None, None, None, 0.0, None, 0, None)
    assert rc == -10
    rc = lib.gpud_launch_streaming_polyphase_stateful_noalloc_cuda(
        None, -1, tp, 16, 2, 8, None, GPUD_NOALLOC_MAX_HISTORY + 1, C.byref(i), C.byref(i), C.byref(d), 0.0, None,
        0, C.byref(i))
    assert rc == -11
