"""SDRIQ001 snapshots over the native reader (gpud_iqfile_*), mirroring
package iqfile (internal/iqfile/iqfile.go): `write`, `read` -> (iq, Meta),
and `Source` -- a looping replay source, paced to the recorded sample rate or
unpaced, whose blocks land in host memory or straight in device memory for
the runner."""
from __future__ import annotations

import ctypes as C
import os
import time
from dataclasses import dataclass

import numpy as np

from . import GPUDError
from ._lib import IQFileMeta, lib


@dataclass
class Meta:
    SampleRate: int
    CenterHz: float
    Samples: int


def _check(rc: int, what: str):
    if rc != 0:
        raise GPUDError(rc, what)


def write(path, iq, sample_rate: int, center_hz: float):
    """iqfile.Write (iqfile.go:33-59)."""
    a = np.ascontiguousarray(iq, dtype=np.complex64)
    _check(lib.gpud_iqfile_write(os.fsencode(path), a.ctypes.data if a.size else None, a.size, int(sample_rate),
                                 float(center_hz)), f"write {path}")


class _File:
    def __init__(self, path):
        self._h = C.c_void_p()
        m = IQFileMeta()
        _check(lib.gpud_iqfile_open(os.fsencode(path), C.byref(self._h), C.byref(m)), f"open {path}")
        self.meta = Meta(int(m.sample_rate), float(m.center_hz), int(m.samples))

    def close(self):
        if self._h:
            lib.gpud_iqfile_close(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        self.close()


def read(path):
    """iqfile.Read (iqfile.go:62-99): (complex64 samples, Meta)."""
    f = _File(path)
    try:
        out = np.zeros(f.meta.Samples, np.complex64)
        if out.size:
            _check(lib.gpud_iqfile_read(f._h, out.ctypes.data, out.size, 0, None), "read")
        return out, f.meta
    finally:
        f.close()


class Source:
    """iqfile.Source (iqfile.go:101-177): replays a snapshot, looping at the
    end.  A paced source reports the samples that have arrived at the recorded
    rate since `start` and not yet been read; an unpaced one the whole file."""

    def __init__(self, path, paced: bool = True):
        self._f = _File(path)
        self.meta = self._f.meta
        self.paced = paced
        self._start = None
        self._delivered = 0

    def start(self):
        self._start = time.monotonic()

    def stop(self):
        pass

    def flush(self):
        pass

    def read_iq(self, n: int, device=None, stream=None):
        """The next n samples: numpy on the host, or a torch complex64 tensor
        on `device` filled by DMA from the mapped file (on `stream`)."""
        if n <= 0:
            return np.zeros(0, np.complex64)
        if device is None:
            out = np.zeros(n, np.complex64)
            _check(lib.gpud_iqfile_read(self._f._h, out.ctypes.data, n, 0, None), "read_iq")
        else:
            import torch
            out = torch.empty(n, dtype=torch.complex64, device=device)
            s = stream if stream is not None else torch.cuda.current_stream(out.device)
            _check(lib.gpud_iqfile_read(self._f._h, out.data_ptr(), n, 1, C.c_void_p(s.cuda_stream)), "read_iq")
        self._delivered += n
        return out

    def buffer_samples(self) -> int:
        """Stats().BufferSamples (iqfile.go:150-170)."""
        if not self.paced or self.meta.SampleRate <= 0 or self._start is None:
            return self.meta.Samples
        arrived = int((time.monotonic() - self._start) * self.meta.SampleRate)
        return max(0, arrived - self._delivered)

    def close(self):
        self._f.close()
