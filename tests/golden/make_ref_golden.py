"""Writes ref_launchers.npz: outputs of the reference's own GPU launchers
(oracle/_ref/libgpudemod_ref.so, the reference's native/exports.cu compiled
from its tree by `make -C oracle ref`) on fixed deterministic inputs, so that
the CPU oracle can be checked against the reference's code without a GPU
(tests/test_golden_ref.py).

Runs on a machine with a CUDA GPU; it loads only the reference library (not
this repository's), and torch for device buffers:

    python tests/golden/make_ref_golden.py [out.npz]

Cases (the inputs are deterministic: the file holds each input's SHA-256,
which the test checks on the inputs it rebuilds):
  * streaming polyphase extraction, gpud_launch_streaming_polyphase_stateful_cuda,
    odd tap counts (the reference's own streaming tests use odd counts):
    (65 taps, D 20, +12.5 kHz), (33, 40, -18.75 kHz), (129, 8, +300 kHz) at
    4 MS/s, one 9000-sample stream cut into chunks of 0, 1, 2, 17, 63, 64, 65,
    129, 511, 2000 and 6148 samples, every chunk's outputs and the carried
    history length, phase count and phase;
  * FM discriminator, gpud_launch_fm_discrim_cuda, on a tone-plus-tones input
    and a two-tone deterministic input of 20000 samples each;
  * the legacy batch slot chain (batch_runner_windows.go:170-178): frequency
    shift from the job's start phase, FIR v2 with the 101-tap low-pass of the
    job's bandwidth, decimation, for two jobs at 2.4 MS/s and two at 10 MS/s
    on 65536 samples (tones 1 kHz inside each passband over a noise-like mix).
"""
import ctypes as C
import hashlib
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle import oracle as O  # noqa: E402  (taps design only: the inputs of the case)
from signals import make_deterministic_iq, make_tone_noise_iq  # noqa: E402

REF_PATH = os.path.join(ROOT, "oracle", "_ref", "libgpudemod_ref.so")
FS = 4_000_000
CHUNKS = [0, 1, 2, 17, 63, 64, 65, 129, 511, 2000, 6148]
STATEFUL = [(65, 20, 12_500.0), (33, 40, -18_750.0), (129, 8, 300_000.0)]
SLOT_N = 1 << 16
SLOTS = [(2_400_000, [(300_000.0, 250_000.0, 300_000, 0.0), (-1_100_000.0, 12_500.0, 48_000, 2.5)]),
         (10_000_000, [(4_300_000.0, 12_500.0, 25_000, -1.0), (1_234_567.0, 250_000.0, 312_500, 0.3)])]


def slot_input(fs, jobs):
    """The slot chain's input: a tone 1 kHz inside each job's passband plus
    the noise-like mix (deterministic)."""
    t = np.arange(SLOT_N, dtype=np.float64)
    x = 0.1 * make_tone_noise_iq(t.size, 0.9).astype(np.complex128)
    for off, _, _, _ in jobs:
        x += np.exp(2j * np.pi * (off + 1000.0) / fs * t)
    return x.astype(np.complex64)


def _ref():
    r = C.CDLL(REF_PATH)
    P, i, d = C.c_void_p, C.c_int, C.c_double
    pi, pd = C.POINTER(C.c_int), C.POINTER(C.c_double)
    r.gpud_stream_sync.restype, r.gpud_stream_sync.argtypes = i, [P]
    r.gpud_launch_fm_discrim_cuda.restype, r.gpud_launch_fm_discrim_cuda.argtypes = i, [P, P, i]
    r.gpud_stream_create.restype, r.gpud_stream_create.argtypes = i, [P]
    r.gpud_stream_destroy.restype, r.gpud_stream_destroy.argtypes = i, [P]
    r.gpud_launch_freq_shift_stream_cuda.restype = i
    r.gpud_launch_freq_shift_stream_cuda.argtypes = [P, P, i, d, d, P]
    r.gpud_launch_fir_v2_stream_cuda.restype, r.gpud_launch_fir_v2_stream_cuda.argtypes = i, [P, P, P, i, i, P]
    r.gpud_launch_decimate_stream_cuda.restype, r.gpud_launch_decimate_stream_cuda.argtypes = i, [P, P, i, i, P]
    f = r.gpud_launch_streaming_polyphase_stateful_cuda
    f.restype, f.argtypes = i, [P, i, P, P, i, i, i, P, P, i, pi, pi, pd, d, P, i, pi]
    return r


def _sha(x):
    return np.frombuffer(hashlib.sha256(np.ascontiguousarray(x).tobytes()).digest(), np.uint8)


def main(out_path):
    import torch
    r = _ref()

    def dev(x):
        return torch.from_numpy(np.ascontiguousarray(x)).cuda()

    def empty(n, dtype):
        return torch.zeros(max(n, 1), dtype=dtype, device="cuda")

    store = {"chunks": np.array(CHUNKS, np.int64), "fs": np.array(FS)}
    x = make_tone_noise_iq(sum(CHUNKS), 0.021)
    store["stateful_in_sha256"] = _sha(x)
    for k, (taps, decim, offset) in enumerate(STATEFUL):
        poly = O.build_polyphase_taps_phase_major(O.base_taps_f32(20_000, FS, taps), decim)
        store[f"stateful{k}_geom"] = np.array([taps, decim, offset])
        store[f"stateful{k}_poly"] = poly
        inc = -2 * math.pi * offset / FS
        cap = taps - 1
        d_taps = dev(poly)
        d_hist, d_scr = empty(cap, torch.complex64), empty(cap, torch.complex64)
        hl, pc, ph, nout = C.c_int(0), C.c_int(0), C.c_double(0.0), C.c_int()
        pos = 0
        for j, n in enumerate(CHUNKS):
            chunk = x[pos:pos + n]
            pos += n
            d_in = dev(chunk) if n else empty(1, torch.complex64)
            d_sh = empty(n, torch.complex64)
            d_out = empty(n // decim + 2, torch.complex64)
            rc = r.gpud_launch_streaming_polyphase_stateful_cuda(
                d_in.data_ptr(), n, d_sh.data_ptr(), d_taps.data_ptr(), poly.size, decim, taps, d_hist.data_ptr(),
                d_scr.data_ptr(), cap, C.byref(hl), C.byref(pc), C.byref(ph), inc, d_out.data_ptr(),
                n // decim + 2, C.byref(nout))
            assert rc == 0, rc
            assert r.gpud_stream_sync(None) == 0
            store[f"stateful{k}_out{j}"] = d_out.cpu().numpy()[: nout.value].copy()
            store[f"stateful{k}_state{j}"] = np.array([hl.value, pc.value, ph.value])
    for k, xin in enumerate((make_tone_noise_iq(20_000, 0.3), make_deterministic_iq(20_000))):
        d_in = dev(xin)
        d_out = empty(xin.size, torch.float32)
        assert r.gpud_launch_fm_discrim_cuda(d_in.data_ptr(), d_out.data_ptr(), xin.size) == 0
        assert r.gpud_stream_sync(None) == 0
        store[f"discrim{k}_in_sha256"] = _sha(xin)
        store[f"discrim{k}_out"] = d_out.cpu().numpy()[: xin.size - 1].copy()
    for g, (fs, jobs) in enumerate(SLOTS):
        x = slot_input(fs, jobs)
        store[f"slot{g}_in_sha256"] = _sha(x)
        d_in = dev(x)
        for j, (off, bw, rate, p0) in enumerate(jobs):
            taps = O.lowpass_fir(max(bw / 2, 200.0), fs, 101).astype(np.float32)
            d_t = dev(taps)
            decim = fs // rate
            n_out = x.size // decim
            sh, flt, dec = (empty(x.size, torch.complex64) for _ in range(3))
            s = C.c_void_p()
            assert r.gpud_stream_create(C.byref(s)) == 0
            assert r.gpud_launch_freq_shift_stream_cuda(d_in.data_ptr(), sh.data_ptr(), x.size,
                                                        -2.0 * math.pi * off / fs, p0, s) == 0
            assert r.gpud_launch_fir_v2_stream_cuda(sh.data_ptr(), flt.data_ptr(), d_t.data_ptr(), x.size, 101, s) == 0
            assert r.gpud_launch_decimate_stream_cuda(flt.data_ptr(), dec.data_ptr(), n_out, decim, s) == 0
            assert r.gpud_stream_sync(s) == 0 and r.gpud_stream_destroy(s) == 0
            store[f"slot{g}_job{j}_out"] = dec.cpu().numpy()[:n_out].copy()
    np.savez_compressed(out_path, **store)
    print("wrote", out_path, os.path.getsize(out_path), "bytes")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "ref_launchers.npz"))
