"""The sixteen drop-in launchers pinned to the reference's own GPU code:
oracle/_ref/libgpudemod_ref.so is the reference's native/exports.cu compiled
from its tree (oracle/Makefile `ref`).  Both libraries run on the same device
inputs and their outputs are compared, launcher by launcher and for the legacy
batch slot chain (freq shift -> FIR v2 -> decimate).

Where this library deliberately differs the bounds say why: its phasors come
from an exact Q0.64 phase (the reference rounds a reduced float64 phase to
float32 before sincosf), its discriminator uses float64 products and atan2
as the reference's CPU path does (the reference kernel: float32), and for an
even tap count its streaming polyphase pair follows the CPU oracle's layout
stride where the reference kernel does not (checked: the reference differs
from the oracle there, this library does not)."""
import ctypes as C
import math
import os

import numpy as np
import pytest

from gpudemod._lib import lib
from oracle import oracle as O
from signals import make_deterministic_iq, make_tone_noise_iq, max_abs, rel_l2

pytestmark = pytest.mark.gpu

REF_PATH = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                        "libgpudemod_ref.so")


@pytest.fixture(scope="module")
def ref(cuda):
    if not os.path.exists(REF_PATH):
        pytest.skip("oracle/_ref/libgpudemod_ref.so not built (needs the reference tree: make -C oracle ref)")
    r = C.CDLL(REF_PATH)
    P, i, d = C.c_void_p, C.c_int, C.c_double
    pi, pd = C.POINTER(C.c_int), C.POINTER(C.c_double)
    sig = {
        "gpud_stream_sync": (i, [P]),
        "gpud_launch_freq_shift_cuda": (i, [P, P, i, d, d]),
        "gpud_launch_freq_shift_stream_cuda": (i, [P, P, i, d, d, P]),
        "gpud_launch_fm_discrim_cuda": (i, [P, P, i]),
        "gpud_upload_fir_taps_cuda": (i, [P, i]),
        "gpud_launch_fir_cuda": (i, [P, P, i, i]),
        "gpud_launch_fir_stream_cuda": (i, [P, P, i, i, P]),
        "gpud_launch_fir_v2_stream_cuda": (i, [P, P, P, i, i, P]),
        "gpud_launch_decimate_cuda": (i, [P, P, i, i]),
        "gpud_launch_decimate_stream_cuda": (i, [P, P, i, i, P]),
        "gpud_launch_am_envelope_cuda": (i, [P, P, i]),
        "gpud_launch_ssb_product_cuda": (i, [P, P, i, d, d]),
        "gpud_launch_streaming_polyphase_prepare_cuda": (i, [P, i, P, i, P, i, i, i, i, d, d, P, pi, pi, pd, P]),
        "gpud_launch_streaming_polyphase_stateful_cuda": (i, [P, i, P, P, i, i, i, P, P, i, pi, pi, pd, d, P, i,
                                                              pi]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(r, name)
        fn.restype, fn.argtypes = res, args
    return r


def dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def empty(n, dtype):
    import torch
    return torch.zeros(max(n, 1), dtype=dtype, device="cuda")


def both(ref, name, *args):
    """Runs one launcher in both libraries; args are callables giving the
    argument list for one library (fresh outputs each)."""
    assert getattr(lib, name)(*args[0]) == 0
    assert getattr(ref, name)(*args[1]) == 0
    assert lib.gpud_stream_sync(None) == 0 and ref.gpud_stream_sync(None) == 0


def test_freq_shift_and_ssb_pinned(ref):
    import torch
    x = make_tone_noise_iq(200_003, 0.013)
    d_in = dev(x)
    for inc, start in ((-0.0123456789, 12345.678), (2.9, -0.5), (0.0, 1.0)):
        a, b = empty(x.size, torch.complex64), empty(x.size, torch.complex64)
        both(ref, "gpud_launch_freq_shift_cuda", (d_in.data_ptr(), a.data_ptr(), x.size, inc, start),
             (d_in.data_ptr(), b.data_ptr(), x.size, inc, start))
        assert max_abs(a.cpu().numpy(), b.cpu().numpy()) <= 2e-6
        h = C.c_void_p()
        assert lib.gpud_stream_create(C.byref(h)) == 0
        a2, b2 = empty(x.size, torch.complex64), empty(x.size, torch.complex64)
        both(ref, "gpud_launch_freq_shift_stream_cuda", (d_in.data_ptr(), a2.data_ptr(), x.size, inc, start, h),
             (d_in.data_ptr(), b2.data_ptr(), x.size, inc, start, h))
        assert lib.gpud_stream_sync(h) == 0 and lib.gpud_stream_destroy(h) == 0
        assert max_abs(a2.cpu().numpy(), b2.cpu().numpy()) <= 2e-6
        fa, fb = empty(x.size, torch.float32), empty(x.size, torch.float32)
        both(ref, "gpud_launch_ssb_product_cuda", (d_in.data_ptr(), fa.data_ptr(), x.size, inc, start),
             (d_in.data_ptr(), fb.data_ptr(), x.size, inc, start))
        assert max_abs(fa.cpu().numpy(), fb.cpu().numpy()) <= 2e-6


def test_discriminator_and_envelope_pinned(ref):
    import torch
    for x in (make_tone_noise_iq(100_000, 0.3), make_deterministic_iq(77_777)):
        d_in = dev(x)
        fa, fb = empty(x.size, torch.float32), empty(x.size, torch.float32)
        both(ref, "gpud_launch_fm_discrim_cuda", (d_in.data_ptr(), fa.data_ptr(), x.size),
             (d_in.data_ptr(), fb.data_ptr(), x.size))
        a, b = fa.cpu().numpy()[: x.size - 1], fb.cpu().numpy()[: x.size - 1]
        # float64 products here, float32 in the reference kernel
        assert max_abs(a, b) <= 2e-6 and rel_l2(a, b) <= 1e-6
        ea, eb = empty(x.size, torch.float32), empty(x.size, torch.float32)
        both(ref, "gpud_launch_am_envelope_cuda", (d_in.data_ptr(), ea.data_ptr(), x.size),
             (d_in.data_ptr(), eb.data_ptr(), x.size))
        assert rel_l2(ea.cpu().numpy(), eb.cpu().numpy()) <= 2e-7


@pytest.mark.parametrize("taps", [2, 33, 101, 256])
def test_fir_and_decimate_pinned(ref, taps):
    import torch
    x = make_tone_noise_iq(70_001, 0.07)
    h = O.lowpass_fir(40_000.0, 2_400_000, taps).astype(np.float32)[:taps]
    d_in, d_h = dev(x), dev(h)
    assert lib.gpud_upload_fir_taps_cuda(h.ctypes.data, taps) == 0
    assert ref.gpud_upload_fir_taps_cuda(h.ctypes.data, taps) == 0
    a, b = empty(x.size, torch.complex64), empty(x.size, torch.complex64)
    both(ref, "gpud_launch_fir_cuda", (d_in.data_ptr(), a.data_ptr(), x.size, taps),
         (d_in.data_ptr(), b.data_ptr(), x.size, taps))
    assert rel_l2(a.cpu().numpy(), b.cpu().numpy()) <= 1e-6
    s = C.c_void_p()
    assert lib.gpud_stream_create(C.byref(s)) == 0
    for name, extra in (("gpud_launch_fir_stream_cuda", ()), ("gpud_launch_fir_v2_stream_cuda", (d_h.data_ptr(),))):
        a, b = empty(x.size, torch.complex64), empty(x.size, torch.complex64)
        args = (lambda out: (d_in.data_ptr(), out.data_ptr(), x.size, taps, s)) if not extra else \
            (lambda out: (d_in.data_ptr(), out.data_ptr(), extra[0], x.size, taps, s))
        both(ref, name, args(a), args(b))
        assert lib.gpud_stream_sync(s) == 0
        assert rel_l2(a.cpu().numpy(), b.cpu().numpy()) <= 1e-6, name
    for factor in (1, 7, 50):
        n_out = x.size // factor
        da, db = empty(n_out, torch.complex64), empty(n_out, torch.complex64)
        both(ref, "gpud_launch_decimate_cuda", (d_in.data_ptr(), da.data_ptr(), n_out, factor),
             (d_in.data_ptr(), db.data_ptr(), n_out, factor))
        assert np.array_equal(da.cpu().numpy(), db.cpu().numpy())
        both(ref, "gpud_launch_decimate_stream_cuda", (d_in.data_ptr(), da.data_ptr(), n_out, factor, s),
             (d_in.data_ptr(), db.data_ptr(), n_out, factor, s))
        assert lib.gpud_stream_sync(s) == 0
        assert np.array_equal(da.cpu().numpy(), db.cpu().numpy())
    assert lib.gpud_stream_destroy(s) == 0


def _run_stateful(f, chunks, poly, decim, taps, inc):
    import torch
    cap = taps - 1
    d_taps = dev(poly)
    d_hist, d_scr = empty(cap, torch.complex64), empty(cap, torch.complex64)
    hl, pc, ph, nout = C.c_int(0), C.c_int(0), C.c_double(0.0), C.c_int()
    outs, states = [], []
    for chunk in chunks:
        n = chunk.size
        d_in = dev(chunk) if n else empty(1, torch.complex64)
        d_sh = empty(n, torch.complex64)
        d_out = empty(n // decim + 2, torch.complex64)
        rc = f(d_in.data_ptr(), n, d_sh.data_ptr(), d_taps.data_ptr(), poly.size, decim, taps, d_hist.data_ptr(),
               d_scr.data_ptr(), cap, C.byref(hl), C.byref(pc), C.byref(ph), inc, d_out.data_ptr(), n // decim + 2,
               C.byref(nout))
        assert rc == 0
        assert lib.gpud_stream_sync(None) == 0
        outs.append(d_out.cpu().numpy()[: nout.value].copy())
        states.append((hl.value, pc.value, ph.value, d_hist.cpu().numpy()[: hl.value].copy()))
    return outs, states


@pytest.mark.parametrize("taps,decim,offset", [(65, 20, 12_500.0), (33, 40, -18_750.0), (129, 8, 300_000.0)])
def test_streaming_stateful_pinned_odd_taps(ref, taps, decim, offset):
    """The reference's own streaming tests use odd tap counts; there both
    libraries apply the same layout and agree chunk by chunk."""
    fs = 4_000_000
    poly = O.build_polyphase_taps_phase_major(O.base_taps_f32(20_000, fs, taps), decim)
    x = make_tone_noise_iq(9000, 0.021)
    sizes = [0, 1, 2, 17, 63, 64, 65, 129, 511, 2000, 6148]
    chunks, pos = [], 0
    for n in sizes:
        chunks.append(x[pos:pos + n])
        pos += n
    inc = -2 * math.pi * offset / fs
    oa, sa = _run_stateful(lib.gpud_launch_streaming_polyphase_stateful_cuda, chunks, poly, decim, taps, inc)
    ob, sb = _run_stateful(ref.gpud_launch_streaming_polyphase_stateful_cuda, chunks, poly, decim, taps, inc)
    for a, b, (ha, pa, fa, hista), (hb, pb, fb, histb) in zip(oa, ob, sa, sb):
        assert a.size == b.size and ha == hb and pa == pb
        assert max_abs(a, b) <= 1e-5
        assert max_abs(hista, histb) <= 2e-6
        assert abs(math.remainder(fa - fb, 2 * math.pi)) <= 1e-9


def test_streaming_stateful_even_taps_follow_the_oracle(ref):
    """Even tap count (the configs' 128 / 256): the reference kernel derives
    its layout stride from num_taps and leaves its own CPU oracle; this
    library stays on the oracle."""
    fs, taps, decim, offset = 2_400_000, 128, 8, 300_000.0
    base = O.base_taps_f32(250_000, fs, taps)  # LowpassFIR makes 129 taps; the oracle applies 128
    poly = O.build_polyphase_taps_phase_major(base, decim)
    x = make_tone_noise_iq(20_000, 0.021)
    chunks = [x[:7001], x[7001:]]
    inc = -2 * math.pi * offset / fs
    oa, _ = _run_stateful(lib.gpud_launch_streaming_polyphase_stateful_cuda, chunks, poly, decim, taps, inc)
    ob, _ = _run_stateful(ref.gpud_launch_streaming_polyphase_stateful_cuda, chunks, poly, decim, taps, inc)
    o_hist, o_ph, o_pc = np.zeros(0, np.complex64), 0.0, 0
    for chunk, a, b in zip(chunks, oa, ob):
        want, o_ph, o_pc, o_hist = O.run_host_core(chunk, fs, offset, o_ph, o_pc, taps, decim, o_hist, poly)
        assert max_abs(a, want) <= 1e-5
        assert rel_l2(b, want) > 1e-3  # the reference kernel's stride disagrees with its oracle


def test_streaming_prepare_pinned(ref):
    import torch
    fs, taps, decim, offset = 4_000_000, 65, 20, 12_500.0
    poly = O.build_polyphase_taps_phase_major(O.base_taps_f32(20_000, fs, taps), decim)
    x = make_deterministic_iq(3000)
    hist = make_tone_noise_iq(taps - 1, 0.05)
    d_in, d_taps, d_hist = dev(x), dev(poly), dev(hist)
    res = []
    for f in (lib.gpud_launch_streaming_polyphase_prepare_cuda, ref.gpud_launch_streaming_polyphase_prepare_cuda):
        d_out = empty(x.size // decim + 2, torch.complex64)
        d_hout = empty(taps - 1, torch.complex64)
        n_out, pc_out, ph_out = C.c_int(), C.c_int(), C.c_double()
        rc = f(d_in.data_ptr(), x.size, d_hist.data_ptr(), taps - 1, d_taps.data_ptr(), poly.size, decim, taps, 3,
               0.7, -2 * math.pi * offset / fs, d_out.data_ptr(), C.byref(n_out), C.byref(pc_out), C.byref(ph_out),
               d_hout.data_ptr())
        assert rc == 0
        assert lib.gpud_stream_sync(None) == 0
        res.append((n_out.value, pc_out.value, ph_out.value, d_out.cpu().numpy()[: n_out.value],
                    d_hout.cpu().numpy()))
    (na, pa, fa, oa, ha), (nb, pb, fb, ob, hb) = res
    assert na == nb and pa == pb
    assert abs(math.remainder(fa - fb, 2 * math.pi)) <= 1e-9
    assert max_abs(oa, ob) <= 1e-5 and max_abs(ha, hb) <= 2e-6


@pytest.mark.parametrize("fs,jobs", [
    (2_400_000, [(300_000.0, 250_000.0, 300_000, 0.0), (-1_100_000.0, 12_500.0, 48_000, 2.5)]),
    (10_000_000, [(4_300_000.0, 12_500.0, 25_000, -1.0), (1_234_567.0, 250_000.0, 312_500, 0.3)]),
])
def test_legacy_batch_chain_pinned(ref, fs, jobs):
    """BatchRunner.ShiftFilterDecimateBatch against the same slot chain
    (batch_runner_windows.go:170-178) run with the reference's launchers."""
    import torch

    import gpudemod as G
    # a tone 1 kHz inside each job's passband, plus the noise-like mix
    t = np.arange(1 << 18, dtype=np.float64)
    x = 0.1 * make_tone_noise_iq(t.size, 0.9).astype(np.complex128)
    for off, _, _, _ in jobs:
        x += np.exp(2j * np.pi * (off + 1000.0) / fs * t)
    x = x.astype(np.complex64)
    br = G.NewBatchRunner(x.size, fs)
    try:
        outs, rates = br.ShiftFilterDecimateBatch(x, [G.ExtractJob(o, b, r, p) for o, b, r, p in jobs])
    finally:
        br.Close()
    d_in = dev(x)
    for (off, bw, rate, p0), got, grate in zip(jobs, outs, rates):
        taps = O.lowpass_fir(max(bw / 2, 200.0), fs, 101).astype(np.float32)
        d_t = dev(taps)
        decim = fs // rate
        n_out = x.size // decim
        sh, flt, dec = (empty(x.size, torch.complex64) for _ in range(3))
        s = C.c_void_p()
        assert lib.gpud_stream_create(C.byref(s)) == 0
        assert ref.gpud_launch_freq_shift_stream_cuda(d_in.data_ptr(), sh.data_ptr(), x.size,
                                                      -2.0 * math.pi * off / fs, p0, s) == 0
        assert ref.gpud_launch_fir_v2_stream_cuda(sh.data_ptr(), flt.data_ptr(), d_t.data_ptr(), x.size, 101, s) == 0
        assert ref.gpud_launch_decimate_stream_cuda(flt.data_ptr(), dec.data_ptr(), n_out, decim, s) == 0
        assert lib.gpud_stream_sync(s) == 0 and lib.gpud_stream_destroy(s) == 0
        want = dec.cpu().numpy()[:n_out]
        assert grate == fs // decim and got.size == want.size
        assert rel_l2(got, want) <= 1e-6
