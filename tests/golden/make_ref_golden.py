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
    and a two-tone deterministic input of 20000 samples each.
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


def _ref():
    r = C.CDLL(REF_PATH)
    P, i, d = C.c_void_p, C.c_int, C.c_double
    pi, pd = C.POINTER(C.c_int), C.POINTER(C.c_double)
    r.gpud_stream_sync.restype, r.gpud_stream_sync.argtypes = i, [P]
    r.gpud_launch_fm_discrim_cuda.restype, r.gpud_launch_fm_discrim_cuda.argtypes = i, [P, P, i]
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
    np.savez_compressed(out_path, **store)
    print("wrote", out_path, os.path.getsize(out_path), "bytes")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "ref_launchers.npz"))
