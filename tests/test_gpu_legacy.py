"""The sixteen reference entry points (native/exports.cu) through the C ABI,
each checked against the oracle or a float64 numpy restatement."""
import ctypes as C
import math

import numpy as np
import pytest

from gpudemod._lib import lib
from oracle import oracle as O
from signals import make_deterministic_iq, make_tone_noise_iq, max_abs, rel_l2

pytestmark = pytest.mark.gpu


def dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def empty(n, dtype):
    import torch
    return torch.zeros(max(n, 1), dtype=dtype, device="cuda")


def sync():
    assert lib.gpud_stream_sync(None) == 0


def test_stream_wrappers(cuda):
    h = C.c_void_p()
    assert lib.gpud_stream_create(C.byref(h)) == 0 and h.value
    assert lib.gpud_stream_sync(h) == 0
    assert lib.gpud_stream_destroy(h) == 0
    assert lib.gpud_stream_create(None) == -1
    assert lib.gpud_stream_destroy(None) == 0


def test_freq_shift(cuda):
    import torch
    x = make_tone_noise_iq(100_003, 0.01)
    inc, start = -0.0123456789, 12345.678
    d_in, d_out = dev(x), empty(x.size, torch.complex64)
    assert lib.gpud_launch_freq_shift_cuda(d_in.data_ptr(), d_out.data_ptr(), x.size, inc, start) == 0
    sync()
    ph = start + inc * np.arange(x.size, dtype=np.float64)
    want = x.astype(np.complex128) * np.exp(1j * ph)
    assert max_abs(d_out.cpu().numpy(), want) <= 2e-6
    assert lib.gpud_launch_freq_shift_cuda(d_in.data_ptr(), d_out.data_ptr(), 0, inc, start) == 0


def test_fm_discrim(cuda):
    import torch
    x = make_tone_noise_iq(50_000, 0.3)
    d_in, d_out = dev(x), empty(x.size, torch.float32)
    assert lib.gpud_launch_fm_discrim_cuda(d_in.data_ptr(), d_out.data_ptr(), x.size) == 0
    sync()
    got = d_out.cpu().numpy()[: x.size - 1]
    assert max_abs(got, O.fm_discrim(x)) <= 1e-6


def _fir_ref(x, taps):
    x = x.astype(np.complex128)
    out = np.zeros(x.size, np.complex128)
    for k, t in enumerate(taps.astype(np.float64)):
        out[k:] += t * x[: x.size - k]
    return out


def test_fir_constant_and_v2(cuda):
    import torch
    x = make_deterministic_iq(70_001)
    taps = O.lowpass_fir(20_000, 200_000, 101).astype(np.float32)
    tp = np.ascontiguousarray(taps)
    assert lib.gpud_upload_fir_taps_cuda(tp.ctypes.data, 101) == 0
    assert lib.gpud_upload_fir_taps_cuda(tp.ctypes.data, 257) == -1
    assert lib.gpud_upload_fir_taps_cuda(None, 10) == -1
    d_in, d_out = dev(x), empty(x.size, torch.complex64)
    assert lib.gpud_launch_fir_cuda(d_in.data_ptr(), d_out.data_ptr(), x.size, 101) == 0
    sync()
    want = _fir_ref(x, taps)
    assert max_abs(d_out.cpu().numpy(), want) <= 1e-5
    d_t = dev(taps)
    d_out2 = empty(x.size, torch.complex64)
    assert lib.gpud_launch_fir_v2_stream_cuda(d_in.data_ptr(), d_out2.data_ptr(), d_t.data_ptr(), x.size, 101,
                                              None) == 0
    sync()
    assert max_abs(d_out2.cpu().numpy(), want) <= 1e-5
    assert lib.gpud_launch_fir_cuda(d_in.data_ptr(), d_out.data_ptr(), x.size, 300) == 0  # no-op beyond 256


def test_decimate_am_ssb(cuda):
    import torch
    x = make_tone_noise_iq(40_000, 0.05)
    d_in = dev(x)
    d_dec = empty(x.size // 7, torch.complex64)
    assert lib.gpud_launch_decimate_cuda(d_in.data_ptr(), d_dec.data_ptr(), x.size // 7, 7) == 0
    d_am = empty(x.size, torch.float32)
    assert lib.gpud_launch_am_envelope_cuda(d_in.data_ptr(), d_am.data_ptr(), x.size) == 0
    d_ssb = empty(x.size, torch.float32)
    inc = 2 * math.pi * 700 / 48_000
    assert lib.gpud_launch_ssb_product_cuda(d_in.data_ptr(), d_ssb.data_ptr(), x.size, inc, 3.0) == 0
    sync()
    assert np.array_equal(d_dec.cpu().numpy(), x[::7][: x.size // 7])
    assert max_abs(d_am.cpu().numpy(), np.abs(x.astype(np.complex128))) <= 1e-6
    ph = 3.0 + inc * np.arange(x.size)
    want = x.real * np.cos(ph) - x.imag * np.sin(ph)
    assert max_abs(d_ssb.cpu().numpy(), want) <= 2e-6


@pytest.mark.parametrize("taps,decim,offset", [(65, 20, 12_500.0), (128, 8, 300_000.0), (33, 40, -18_750.0)])
def test_streaming_polyphase_stateful_matches_oracle(cuda, taps, decim, offset):
    import torch
    fs = 4_000_000 if decim != 8 else 2_400_000
    base = O.base_taps_f32(20_000 if decim != 8 else 250_000, fs, taps)
    poly = O.build_polyphase_taps_phase_major(base, decim)
    cap = taps - 1
    d_taps = dev(poly)
    d_hist, d_scr = empty(cap, torch.complex64), empty(cap, torch.complex64)
    hl, pc, ph = C.c_int(0), C.c_int(0), C.c_double(0.0)
    nout = C.c_int()
    inc = -2 * math.pi * offset / fs
    o_hist, o_ph, o_pc = np.zeros(0, np.complex64), 0.0, 0
    x = make_tone_noise_iq(9000, 0.021)
    pos = 0
    for n in [0, 1, 2, 17, 63, 64, 65, 129, 511, 2000, 6148]:
        chunk = x[pos:pos + n]
        pos += n
        d_in = dev(chunk) if n else empty(1, torch.complex64)
        d_sh = empty(n, torch.complex64)
        d_out = empty(n // decim + 2, torch.complex64)
        rc = lib.gpud_launch_streaming_polyphase_stateful_cuda(
            d_in.data_ptr(), n, d_sh.data_ptr(), d_taps.data_ptr(), poly.size, decim, taps, d_hist.data_ptr(),
            d_scr.data_ptr(), cap, C.byref(hl), C.byref(pc), C.byref(ph), inc, d_out.data_ptr(), n // decim + 2,
            C.byref(nout))
        assert rc == 0
        sync()
        want, o_ph, o_pc, o_hist = O.run_host_core(chunk, fs, offset, o_ph, o_pc, taps, decim, o_hist, poly)
        assert nout.value == want.size and pc.value == o_pc and hl.value == o_hist.size
        assert max_abs(d_out.cpu().numpy()[: nout.value], want) <= 1e-5
        assert max_abs(d_hist.cpu().numpy()[: hl.value], o_hist) <= 1e-5
        d = ph.value - o_ph
        assert abs(math.remainder(d, 2 * math.pi)) <= 1e-9


def test_streaming_polyphase_stateful_error_codes(cuda):
    i = C.c_int(0)
    d = C.c_double(0)
    f = lib.gpud_launch_streaming_polyphase_stateful_cuda
    assert f(None, 0, None, None, 10, 2, 5, None, None, 4, None, C.byref(i), C.byref(d), 0.0, None, 0,
             C.byref(i)) == -10
    assert f(None, -1, None, 1, 10, 2, 5, None, None, 4, C.byref(i), C.byref(i), C.byref(d), 0.0, None, 0,
             C.byref(i)) == -11
    assert f(None, 0, None, 1, 4, 2, 5, None, None, 4, C.byref(i), C.byref(i), C.byref(d), 0.0, None, 0,
             C.byref(i)) == -12
    assert f(None, 5, None, 1, 6, 2, 5, None, None, 4, C.byref(i), C.byref(i), C.byref(d), 0.0, None, 0,
             C.byref(i)) == -13


def test_streaming_polyphase_prepare_matches_oracle(cuda):
    import torch
    fs, taps, decim, offset = 4_000_000, 65, 20, 12_500.0
    base = O.base_taps_f32(20_000, fs, taps)
    poly = O.build_polyphase_taps_phase_major(base, decim)
    x = make_deterministic_iq(3000)
    want, w_ph, w_pc, w_hist = O.run_host_core(x, fs, offset, 0.7, 3, taps, decim, np.zeros(0, np.complex64), poly)
    d_in, d_taps = dev(x), dev(poly)
    d_out = empty(x.size // decim + 2, torch.complex64)
    d_hout = empty(taps - 1, torch.complex64)
    n_out, pc_out, ph_out = C.c_int(), C.c_int(), C.c_double()
    rc = lib.gpud_launch_streaming_polyphase_prepare_cuda(
        d_in.data_ptr(), x.size, None, 0, d_taps.data_ptr(), poly.size, decim, taps, 3, 0.7,
        -2 * math.pi * offset / fs, d_out.data_ptr(), C.byref(n_out), C.byref(pc_out), C.byref(ph_out),
        d_hout.data_ptr())
    assert rc == 0
    sync()
    assert n_out.value == want.size and pc_out.value == w_pc
    assert max_abs(d_out.cpu().numpy()[: want.size], want) <= 1e-5
    assert max_abs(d_hout.cpu().numpy()[: w_hist.size], w_hist) <= 1e-5
    assert abs(math.remainder(ph_out.value - w_ph, 2 * math.pi)) <= 1e-9
