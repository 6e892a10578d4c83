"""gpudemod -- Python mirror of the reference's Go package
`internal/demod/gpudemod` over libgpudemod_kernels.so.

Same names and argument meaning as the Go API (gpudemod.go, batch_runner.go,
streaming_types.go, streaming_gpu_stub.go), so tests read like the
reference's own: `NewBatchRunner(maxSamples, sampleRate)`,
`runner.StreamingExtractGPU(iq, jobs)`, `ExactIntegerDecimation`, ...  Plus
`ChannelRunner`, the batched / serving runner (admit / retire / process_block
/ results / stats / snapshot).

All compute runs in the CUDA library; nothing here falls back to the CPU.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._lib import AutotuneEntry, BatchAudioResult, RDSJob, RDSResult, SegmentAudioResult, ChannelResult, ChannelSpec, PilotJob, PilotResult, RunnerStats, StageTime, lib

# DemodType (gpudemod.go:69-76) -> runner modes
DemodNFM, DemodWFM, DemodAM, DemodUSB, DemodLSB, DemodCW = range(6)
MODE_IQ, MODE_NFM, MODE_WFM, MODE_WFM_STEREO, MODE_AM, MODE_USB, MODE_LSB, MODE_CW = range(8)
MODE_BY_NAME = {"IQ": MODE_IQ, "NFM": MODE_NFM, "WFM": MODE_WFM, "WFM_STEREO": MODE_WFM_STEREO, "AM": MODE_AM,
                "USB": MODE_USB, "LSB": MODE_LSB, "CW": MODE_CW}
CH_EMIT_IQ, CH_RDS, CH_AUDIO48K, CH_DEEMPH75, CH_NO_DEEMPH = 1, 2, 4, 8, 16
CH_PCM_F32, CH_BATCH_STEREO, CH_FREE_STEREO = 32, 64, 128
FORM_DENSE, FORM_WIDE, FORM_GROUP, FORM_MOD = 0, 1, 2, 3
SCHED_BATCHED, SCHED_PLAIN = 0, 1

E_ARG, E_DECIM, E_TAPS, E_BUDGET, E_SLOTS, E_SLOT, E_BLOCK, E_TIMEOUT, E_CUDA, E_MODE, E_DEVICE_STATUS, E_STATE = \
    -20, -21, -22, -23, -24, -25, -26, -27, -28, -29, -30, -31


class ErrUnavailable(RuntimeError):
    """gpudemod.ErrUnavailable (errors.go)."""


class GPUDError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"gpudemod error {code}: {msg}")
        self.code = code


def Available() -> bool:
    """gpudemod.Available (gpudemod.go:95-101)."""
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:  # pragma: no cover
        return False


def ExactIntegerDecimation(sample_rate: int, out_rate: int) -> int:
    """cpu_oracle.go:155-163."""
    if sample_rate <= 0 or out_rate <= 0:
        raise ValueError(f"invalid sampleRate/outRate: {sample_rate}/{out_rate}")
    if sample_rate % out_rate != 0:
        raise ValueError(f"streaming polyphase extractor requires integer decimation: "
                         f"sampleRate={sample_rate} outRate={out_rate}")
    return sample_rate // out_rate


def StreamingConfigHash(signal_id: int, offset_hz: float, bandwidth: float, out_rate: int, num_taps: int,
                        sample_rate: int) -> int:
    """streaming_types.go:58-72 (offset and bandwidth are not hashed)."""
    return int(lib.gpud_streaming_config_hash(int(signal_id), int(out_rate), int(num_taps), int(sample_rate)))


def BuildPolyphaseTapsPhaseMajor(base, decim: int) -> np.ndarray:
    """polyphase.go:6-20: out[p*L + k] = base[p + k*D], L = ceil(len/D)."""
    base = np.asarray(base, dtype=np.float32)
    if decim <= 0 or base.size == 0:
        return np.zeros(0, np.float32)
    L = (base.size + decim - 1) // decim
    out = np.zeros(decim * L, np.float32)
    for p in range(decim):
        src = p + decim * np.arange(L)
        ok = src < base.size
        out[p * L: p * L + L][ok] = base[src[ok]]
    return out


@dataclass
class StreamingExtractJob:
    SignalID: int
    OffsetHz: float
    Bandwidth: float
    OutRate: int
    NumTaps: int
    ConfigHash: int


@dataclass
class StreamingExtractResult:
    SignalID: int
    IQ: np.ndarray
    Rate: int
    NOut: int
    PhaseCount: int
    HistoryLen: int
    NCOPhase: float = 0.0


def _check(r, rc: int):
    if rc != 0:
        msg = lib.gpud_runner_last_error(r).decode() if r else ""
        raise GPUDError(rc, msg)


def _spec(signal_id, offset_hz, bandwidth, out_rate, num_taps, config_hash=0, mode=MODE_IQ, flags=0,
          demod_decim=1) -> ChannelSpec:
    return ChannelSpec(int(signal_id), float(offset_hz), float(bandwidth), int(out_rate), int(num_taps),
                       int(config_hash) & ((1 << 64) - 1), int(mode), int(flags), int(demod_decim), 0)


def _iq_ptr(iq):
    """(pointer, n, on_device, keepalive) for numpy (host) or torch (host or cuda)."""
    try:
        import torch
        if isinstance(iq, torch.Tensor):
            t = iq.contiguous()
            if t.dtype != torch.complex64:
                t = t.to(torch.complex64)
            return t.data_ptr(), t.numel(), 1 if t.is_cuda else 0, t
    except ImportError:  # pragma: no cover
        pass
    a = np.ascontiguousarray(iq, dtype=np.complex64)
    return (a.ctypes.data if a.size else None), a.size, 0, a


class ChannelRunner:
    """Batched / serving runner (gpud_runner_*): device-resident channel slots,
    one launch sequence per IQ block for all channels."""

    def __init__(self, sample_rate: int, max_block: int, max_channels: int = 64, max_taps: int = 1024,
                 device_mem_budget: int = 0):
        self._r = C.c_void_p()
        rc = lib.gpud_runner_create(int(sample_rate), int(max_block), int(max_channels), int(max_taps),
                                    int(device_mem_budget), C.byref(self._r))
        if rc != 0:
            raise GPUDError(rc, "gpud_runner_create failed")
        self.sample_rate = sample_rate
        self.max_block = max_block

    # -- lifecycle ---------------------------------------------------------
    def close(self):
        if self._r:
            lib.gpud_runner_destroy(self._r)  # waits for every block in flight
            self._r = C.c_void_p()
        self._keep = ()  # the blocks in flight no longer need their inputs

    Close = close

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def admit(self, signal_id, offset_hz, bandwidth, out_rate, num_taps=101, mode=MODE_IQ, flags=0,
              config_hash=0, demod_decim=1) -> int:
        """Admits a channel.  demod_decim > 1 adds the pre-demod decimating
        low-pass (recorder/streamer.go:1098-1146): extraction runs at
        out_rate, the demodulator at out_rate // demod_decim."""
        slot = C.c_int()
        spec = _spec(signal_id, offset_hz, bandwidth, out_rate, num_taps, config_hash, mode, flags, demod_decim)
        _check(self._r, lib.gpud_runner_admit(self._r, C.byref(spec), C.byref(slot)))
        return slot.value

    def footprint(self, out_rate, mode=MODE_IQ, flags=0, num_taps=101, demod_decim=1) -> int:
        b = C.c_uint64()
        spec = _spec(0, 0, 0, out_rate, num_taps, 0, mode, flags, demod_decim)
        _check(self._r, lib.gpud_runner_channel_footprint(self._r, C.byref(spec), C.byref(b)))
        return b.value

    def retire(self, slot: int):
        _check(self._r, lib.gpud_runner_retire(self._r, int(slot)))

    def update(self, slot: int, offset_hz: float, bandwidth: float):
        _check(self._r, lib.gpud_runner_update(self._r, int(slot), float(offset_hz), float(bandwidth)))

    def set_autotune_table(self, entries):
        """entries: (taps, decim, form, group_phases) overrides of the
        extraction form per channel class (gpud_runner_set_autotune_table)."""
        arr = (AutotuneEntry * max(1, len(entries)))(*[AutotuneEntry(*map(int, e)) for e in entries])
        _check(self._r, lib.gpud_runner_set_autotune_table(self._r, arr, len(entries)))

    def set_channel_groups(self, enable: bool):
        """Tensor-core channel groups on (default) or off
        (gpud_runner_set_channel_groups); off keeps every channel's output
        bit-identical alone and in any mix."""
        _check(self._r, lib.gpud_runner_set_channel_groups(self._r, 1 if enable else 0))

    def channel_form(self, slot: int):
        """(form, phases per group, groups) of an admitted channel."""
        f, pg, ng = C.c_int(), C.c_int(), C.c_int()
        _check(self._r, lib.gpud_runner_channel_form(self._r, int(slot), C.byref(f), C.byref(pg), C.byref(ng)))
        return f.value, pg.value, ng.value

    def set_schedule(self, schedule: int):
        _check(self._r, lib.gpud_runner_set_schedule(self._r, int(schedule)))

    # -- blocks ------------------------------------------------------------
    def process_block(self, iq):
        ptr, n, dev, keep = _iq_ptr(iq)
        _check(self._r, lib.gpud_runner_process_block(self._r, ptr, n, dev))
        del keep

    def submit(self, iq) -> int:
        ptr, n, dev, keep = _iq_ptr(iq)
        t = C.c_uint64()
        _check(self._r, lib.gpud_runner_submit(self._r, ptr, n, dev, C.byref(t)))
        # three blocks may be in flight: keep their inputs alive
        self._keep = (getattr(self, "_keep", (None, None, None)) + (keep,))[-3:]
        return t.value

    def wait(self, ticket: int, timeout_ms: int = 10000):
        _check(self._r, lib.gpud_runner_wait(self._r, int(ticket), int(timeout_ms)))

    def result(self, slot: int, payload: bool = True) -> dict:
        """Results of the most recently completed block.  With payload=False (required while host
        outputs are off: the payload pointers are then device pointers) only
        counts, flags and margins are returned."""
        res = ChannelResult()
        _check(self._r, lib.gpud_runner_result(self._r, int(slot), C.byref(res)))

        def arr(ptr, n, dt, width):
            if not payload or not ptr or n <= 0:
                return np.zeros(0, dt)
            buf = (C.c_float * (n * width)).from_address(C.addressof(ptr.contents))
            return np.frombuffer(buf, dtype=np.float32).view(dt).copy()

        pcm = np.zeros(0, np.int16)
        if payload and res.pcm and res.n_pcm > 0:
            buf = (C.c_int16 * res.n_pcm).from_address(C.addressof(res.pcm.contents))
            pcm = np.frombuffer(buf, dtype=np.int16).copy()
        elif payload and res.pcm_f32 and res.n_pcm > 0:
            buf = (C.c_float * res.n_pcm).from_address(C.addressof(res.pcm_f32.contents))
            pcm = np.frombuffer(buf, dtype=np.float32).copy()
        return {
            "pcm": pcm,
            "pcm_rate": res.pcm_rate,
            "signal_id": res.signal_id,
            "rate": res.rate,
            "n_iq": res.n_iq,
            "phase_count": res.phase_count,
            "history_len": res.history_len,
            "nco_phase": res.nco_phase,
            "iq": arr(res.iq, res.n_iq, np.complex64, 2),
            "audio": arr(res.audio, res.n_audio, np.float32, 1),
            "audio_channels": res.audio_channels,
            "rds": arr(res.rds, res.n_rds, np.complex64, 2),
            "rds_rate": res.rds_rate,
            "locked": bool(res.flags & 1),
            "stereo": bool(res.flags & 2),
            "coherence": res.coherence,
            "pilot_hz": res.pilot_hz,
            "err_avg": res.err_avg,
            "pll_path": res.pll_path,
            "pll_iters": res.pll_iters,
        }

    def reset_stats(self):
        """Clear the block-latency window (p50 / p99)."""
        _check(self._r, lib.gpud_runner_reset_stats(self._r))

    def stats(self) -> dict:
        s = RunnerStats()
        _check(self._r, lib.gpud_runner_stats_get(self._r, C.byref(s)))
        return {f: getattr(s, f) for f, _ in RunnerStats._fields_}

    def set_host_outputs(self, on: bool):
        _check(self._r, lib.gpud_runner_set_host_outputs(self._r, 1 if on else 0))

    def set_pll_solver(self, parallel: bool, max_iters: int = 0):
        """parallel=False: serial loop only.  max_iters > 1 caps the Newton
        iterations before a block falls back to the serial loop."""
        v = 0 if not parallel else (int(max_iters) if max_iters > 1 else 1)
        _check(self._r, lib.gpud_runner_set_pll_solver(self._r, v))

    def set_profiling(self, on: bool):
        _check(self._r, lib.gpud_runner_set_profiling(self._r, 1 if on else 0))

    def stage_times(self) -> list:
        arr = (StageTime * 64)()
        cnt = C.c_int()
        _check(self._r, lib.gpud_runner_stage_times(self._r, arr, 64, C.byref(cnt)))
        return [(arr[i].name.decode(), arr[i].ms) for i in range(min(cnt.value, 64))]

    def stream_handle(self) -> int:
        h = C.c_void_p()
        _check(self._r, lib.gpud_runner_stream(self._r, C.byref(h)))
        return h.value or 0

    def snapshot(self, slot: int) -> bytes:
        n = C.c_uint64()
        _check(self._r, lib.gpud_runner_snapshot(self._r, int(slot), None, C.byref(n)))
        buf = C.create_string_buffer(n.value)
        _check(self._r, lib.gpud_runner_snapshot(self._r, int(slot), buf, C.byref(n)))
        return buf.raw[: n.value]

    def restore(self, slot: int, blob: bytes):
        buf = C.create_string_buffer(blob, len(blob))
        _check(self._r, lib.gpud_runner_restore(self._r, int(slot), buf, len(blob)))

    # -- BatchRunner.StreamingExtractGPU ----------------------------------
    def streaming_extract(self, iq, jobs):
        a = np.ascontiguousarray(iq, dtype=np.complex64)
        specs = (ChannelSpec * max(1, len(jobs)))()
        for i, j in enumerate(jobs):
            specs[i] = _spec(j.SignalID, j.OffsetHz, j.Bandwidth, j.OutRate, j.NumTaps, j.ConfigHash)
        results = (ChannelResult * max(1, len(jobs)))()
        cap = sum(a.size // max(1, self.sample_rate // max(1, j.OutRate)) + 2 for j in jobs) + 16
        out = np.zeros(cap, np.complex64)
        rc = lib.gpud_runner_streaming_extract(self._r, a.ctypes.data if a.size else None, a.size, specs,
                                               len(jobs), results, out.ctypes.data, cap)
        _check(self._r, rc)
        outs, pos = [], 0
        for i, j in enumerate(jobs):
            r = results[i]
            iqo = out[pos: pos + r.n_iq].copy()
            pos += r.n_iq
            outs.append(StreamingExtractResult(j.SignalID, iqo, r.rate, r.n_iq, r.phase_count, r.history_len,
                                               r.nco_phase))
        return outs


class BatchRunner:
    """gpudemod.BatchRunner (batch_runner.go:12-98) -- streaming extraction
    keyed by SignalID with per-signal state on the device."""

    def __init__(self, max_samples: int, sample_rate: int, max_channels: int = 256, max_taps: int = 1024):
        self._cr = ChannelRunner(sample_rate, max(1, max_samples), max_channels, max_taps)
        self.sampleRate = sample_rate
        self._slots, self._slot_n, self._d_in = [], 0, None

    def StreamingExtractGPU(self, iq_new, jobs):
        """streaming_gpu_stub.go:21-26."""
        if self._cr is None:
            raise ErrUnavailable("gpudemod batch runner unavailable")
        return self._cr.streaming_extract(iq_new, jobs)

    StreamingExtractGPUExec = StreamingExtractGPU

    def ResetSignalState(self, signal_id: int):
        """stream_state.go:9-16: forget one signal (its next job starts fresh)."""
        _check(self._cr._r, lib.gpud_runner_reset_signal(self._cr._r, int(signal_id)))

    def ResetAllSignalStates(self):
        """stream_state.go:18-24."""
        _check(self._cr._r, lib.gpud_runner_reset_all_signals(self._cr._r))

    def ShiftFilterDecimateBatch(self, iq, jobs):
        """batch_runner.go:61-68 with the GPU slot path of
        batch_runner_windows.go:99-182: one H2D of the block; per job on its
        own stream the shift from job.PhaseStart (phase PhaseStart + i*inc),
        the 101-tap FIR (LowpassFIR(max(BW/2, 200)) as float32, zero history)
        and the decimation by the exact integer factor (len(iq) // D outputs);
        then each stream is synchronised and its output copied back.
        Returns (outs, rates)."""
        import torch
        if self._cr is None:
            raise ErrUnavailable("gpudemod batch runner unavailable")
        n = len(iq)
        outs, rates = [None] * len(jobs), [0] * len(jobs)
        if n == 0:
            return outs, rates
        self._alloc_slots(len(jobs), n)
        self._d_in[:n].copy_(torch.as_tensor(np.ascontiguousarray(iq, np.complex64)))
        n_outs = []
        for i, job in enumerate(jobs):
            buf = self._slots[i]
            taps = LowpassFIR(max(job.BW / 2, 200.0), self.sampleRate, 101).astype(np.float32)
            buf["taps"][:taps.size].copy_(torch.from_numpy(taps))
            decim = ExactIntegerDecimation(self.sampleRate, job.OutRate)
            n_out = n // decim
            if n_out <= 0:
                raise ValueError("not enough output samples after decimation")
            inc = -2.0 * np.pi * job.OffsetHz / self.sampleRate
            torch.cuda.current_stream().synchronize()  # the block and taps copies have landed
            s = buf["stream"]
            for rc, what in ((lib.gpud_launch_freq_shift_stream_cuda(self._d_in.data_ptr(), buf["sh"].data_ptr(), n,
                                                                     inc, float(job.PhaseStart), s), "freq shift"),
                             (lib.gpud_launch_fir_v2_stream_cuda(buf["sh"].data_ptr(), buf["flt"].data_ptr(),
                                                                 buf["taps"].data_ptr(), n, taps.size, s), "FIR v2"),
                             (lib.gpud_launch_decimate_stream_cuda(buf["flt"].data_ptr(), buf["dec"].data_ptr(),
                                                                   n_out, decim, s), "decimate")):
                if rc != 0:
                    raise RuntimeError(f"gpu {what} failed ({rc})")
            n_outs.append(n_out)
            rates[i] = self.sampleRate // decim
        for i, n_out in enumerate(n_outs):
            rc = lib.gpud_stream_sync(self._slots[i]["stream"])
            if rc != 0:
                raise RuntimeError(f"cuda stream sync failed ({rc})")
            outs[i] = self._slots[i]["dec"][:n_out].cpu().numpy()
        return outs, rates

    def ShiftFilterDecimateBatchWithPhase(self, iq, jobs):
        """batch_runner.go:72-98: ExtractResults with PhaseEnd = PhaseStart +
        inc * len(iq)."""
        outs, rates = self.ShiftFilterDecimateBatch(iq, jobs)
        res = []
        for i, job in enumerate(jobs):
            inc = -2.0 * np.pi * job.OffsetHz / self.sampleRate
            res.append(ExtractResult(outs[i], rates[i], job.PhaseStart + inc * len(iq)))
        return res

    def _alloc_slots(self, count: int, n: int):
        """Per-slot device buffers and streams (batch_runner_windows.go:58-97):
        reallocated when the slot count changes or the block grows."""
        import torch
        if len(self._slots) == count and n <= self._slot_n:
            return
        self._free_slots()
        dev = torch.device("cuda", torch.cuda.current_device())
        self._d_in = torch.empty(n, dtype=torch.complex64, device=dev)
        for _ in range(count):
            h = C.c_void_p()
            rc = lib.gpud_stream_create(C.byref(h))
            if rc != 0:
                raise RuntimeError(f"cudaStreamCreate failed ({rc})")
            self._slots.append({"sh": torch.empty(n, dtype=torch.complex64, device=dev),
                                "flt": torch.empty(n, dtype=torch.complex64, device=dev),
                                "dec": torch.empty(n, dtype=torch.complex64, device=dev),
                                "taps": torch.empty(256, dtype=torch.float32, device=dev), "stream": h})
        self._slot_n = n

    def _free_slots(self):
        for sl in self._slots:
            lib.gpud_stream_destroy(sl["stream"])
        self._slots, self._slot_n, self._d_in = [], 0, None

    def Close(self):
        self._free_slots()
        if self._cr is not None:
            self._cr.close()
            self._cr = None


@dataclass
class ExtractJob:
    """gpudemod.ExtractJob (batch.go:5-10)."""
    OffsetHz: float
    BW: float
    OutRate: int
    PhaseStart: float = 0.0


@dataclass
class ExtractResult:
    """gpudemod.ExtractResult (batch.go:14-18)."""
    IQ: np.ndarray
    Rate: int
    PhaseEnd: float


def _go_round(x: float) -> int:
    """math.Round for x >= 0: half away from zero (x - floor(x) is exact)."""
    f = int(np.floor(x))
    return f + 1 if x - f >= 0.5 else f


def LowpassFIR(cutoff_hz: float, sample_rate: int, taps: int) -> np.ndarray:
    """dsp.LowpassFIR (dsp/fir.go:6-28), float64, odd length."""
    out = np.zeros((taps | 1) + 1, np.float64)
    n = lib.gpud_lowpass_fir(float(cutoff_hz), int(sample_rate), int(taps),
                             out.ctypes.data_as(C.POINTER(C.c_double)), out.size)
    if n < 0:
        raise ValueError(f"LowpassFIR({cutoff_hz}, {sample_rate}, {taps}) rejected: {n}")
    return out[:n]


class Engine:
    """gpudemod.Engine (gpudemod.go:81-489): the single-signal shift / FIR /
    decimate / demod engine, every stage on the device.

    ShiftFilterDecimate and the front end of Demod give the results the
    reference keeps: its CPU dsp chain (FreqShift from phase 0, incremented
    before use; zero-history FIR with float64 accumulation; Decimate keeping
    every D-th sample from index 0), here on the device through
    gpud_shift_fir_decimate_cuda.  Demod's FIR taps are set on the first call
    (101 taps of LowpassFIR(max(bw/2, 200))) and kept, as SetFIR keeps them;
    the demodulators are the drop-in launchers: the discriminator, the AM
    envelope without mean removal, and the BFO product whose phase advances
    by 2*pi*bfo/sampleRate per decimated sample and carries across calls
    (gpudemod.go:296-318)."""

    def __init__(self, max_samples: int, sample_rate: int):
        """gpudemod.New (gpudemod.go:103-150)."""
        if max_samples <= 0:
            raise ValueError("invalid maxSamples")
        if sample_rate <= 0:
            raise ValueError("invalid sampleRate")
        if not Available():
            raise ErrUnavailable("cuda device not available")
        import torch
        self.maxSamples, self.sampleRate = int(max_samples), int(sample_rate)
        self.phase = 0.0
        self.bfoPhase = 0.0
        self.firTaps = None
        self._dev = torch.device("cuda", torch.cuda.current_device())
        self._in = torch.empty(self.maxSamples, dtype=torch.complex64, device=self._dev)
        self._sh = torch.empty_like(self._in)
        self._dec = torch.empty_like(self._in)
        self._audio = torch.empty(self.maxSamples, dtype=torch.float32, device=self._dev)
        self._taps = torch.empty(256, dtype=torch.float64, device=self._dev)
        self.cudaReady = True
        self._last_shift = self._last_demod = False

    def SetFIR(self, taps):
        """gpudemod.go:152-164: at most 256 float32 taps, uploaded to the
        launchers' constant taps as well."""
        t = np.asarray(taps, np.float32)[:256]
        if t.size == 0:
            self.firTaps = None
            return
        self.firTaps = t.copy()
        if self.cudaReady:
            lib.gpud_upload_fir_taps_cuda(self.firTaps.ctypes.data, self.firTaps.size)

    def LastShiftUsedGPU(self) -> bool:
        return self._last_shift

    def LastDemodUsedGPU(self) -> bool:
        return self._last_demod

    def _front(self, iq, offset_hz: float, taps64: np.ndarray, decim: int):
        """Shift, FIR and decimate on the device; returns the count."""
        import torch
        x = torch.as_tensor(np.ascontiguousarray(iq, np.complex64))
        n = x.numel()
        if n > self.maxSamples:
            raise ValueError("sample count exceeds engine capacity")
        self._in[:n].copy_(x)
        self._taps[:taps64.size].copy_(torch.from_numpy(np.ascontiguousarray(taps64, np.float64)))
        cnt = C.c_int()
        rc = lib.gpud_shift_fir_decimate_cuda(self._in.data_ptr(), n, self.sampleRate, float(offset_hz),
                                              self._taps.data_ptr(), taps64.size, int(decim), self._sh.data_ptr(),
                                              self._dec.data_ptr(), self.maxSamples, C.byref(cnt), None)
        if rc != 0:
            raise GPUDError(rc, "shift/FIR/decimate launch failed")
        return cnt.value

    def ShiftFilterDecimate(self, iq, offset_hz: float, bw: float, out_rate: int):
        """gpudemod.go:325-350: (IQ, rate) with cutoff BW/2 clamped to
        [200, fs/2 - 1], 101 taps, decimation round(fs / out_rate)."""
        if len(iq) == 0:
            return None, 0
        if out_rate <= 0:
            raise ValueError("invalid output sample rate")
        cutoff = min(max(bw / 2, 200.0), self.sampleRate / 2 - 1)
        decim = max(1, _go_round(self.sampleRate / out_rate))
        n = self._front(iq, offset_hz, LowpassFIR(cutoff, self.sampleRate, 101), decim)
        self._last_shift = True
        import torch
        torch.cuda.synchronize(self._dev)
        return self._dec[:n].cpu().numpy(), self.sampleRate // decim

    def Demod(self, iq, offset_hz: float, bw: float, mode: int):
        """gpudemod.go:356-461: (audio, demod input rate)."""
        if not self.cudaReady:
            raise RuntimeError("cuda demod engine is not initialized")
        if len(iq) == 0:
            return None, 0
        if len(iq) > self.maxSamples:
            raise ValueError("sample count exceeds engine capacity")
        if mode in (DemodNFM, DemodAM, DemodUSB, DemodLSB, DemodCW):
            out_rate = 48000
        elif mode == DemodWFM:
            out_rate = 192000
        else:
            raise ValueError("unsupported demod type")
        if self.firTaps is None:
            self.SetFIR(LowpassFIR(max(bw / 2, 200.0), self.sampleRate, 101).astype(np.float32))
        decim = max(1, _go_round(self.sampleRate / out_rate))
        m = self._front(iq, offset_hz, self.firTaps.astype(np.float64), decim)
        self.phase += -2.0 * np.pi * offset_hz / self.sampleRate * len(iq)
        self._last_shift = True
        rate = self.sampleRate // decim
        dec, audio = self._dec.data_ptr(), self._audio.data_ptr()
        if mode in (DemodNFM, DemodWFM):
            rc, cnt = lib.gpud_launch_fm_discrim_cuda(dec, audio, m), max(0, m - 1)
        elif mode == DemodAM:
            rc, cnt = lib.gpud_launch_am_envelope_cuda(dec, audio, m), m
        else:
            bfo = -700.0 if mode == DemodLSB else 700.0
            inc = 2.0 * np.pi * bfo / self.sampleRate
            rc, cnt = lib.gpud_launch_ssb_product_cuda(dec, audio, m, inc, self.bfoPhase), m
            self.bfoPhase += inc * m
        if rc != 0:
            raise GPUDError(rc, "demod launch failed")
        self._last_demod = True
        import torch
        torch.cuda.synchronize(self._dev)
        return self._audio[:cnt].cpu().numpy(), rate

    DemodFused = Demod  # gpudemod.go:352-354

    def ShiftFilterDecimateBatch(self, iq, jobs):
        """batch.go:20-32: ShiftFilterDecimate per job."""
        outs, rates = [], []
        for job in jobs:
            o, r = self.ShiftFilterDecimate(iq, job.OffsetHz, job.BW, job.OutRate)
            outs.append(o)
            rates.append(r)
        return outs, rates

    def ShiftFilterDecimateBatchWithPhase(self, iq, jobs):
        """batch.go:36-50: PhaseEnd = PhaseStart + inc * len(iq)."""
        res = []
        for job in jobs:
            o, r = self.ShiftFilterDecimate(iq, job.OffsetHz, job.BW, job.OutRate)
            inc = -2.0 * np.pi * job.OffsetHz / self.sampleRate
            res.append(ExtractResult(o, r, job.PhaseStart + inc * len(iq)))
        return res

    def Close(self):
        self._in = self._sh = self._dec = self._audio = self._taps = None
        self.firTaps = None
        self.cudaReady = False


def NewBatchRunner(max_samples: int, sample_rate: int) -> BatchRunner:
    """batch_runner.go:23-35."""
    return BatchRunner(max_samples, sample_rate)


def kernel_launch_count() -> int:
    return int(lib.gpud_kernel_launch_count())


class StereoPilotDetector:
    """classifier.StereoPilotPresent / estimateWFMPilot (internal/classifier/
    pll.go:75-131) for a batch of FM-multiplex basebands on the device
    (gpud_pilot_*).  Inputs are CUDA tensors (complex64) or host arrays, which
    are copied to the device first."""

    def __init__(self, max_jobs: int = 64, max_samples: int = 1 << 20):
        self._p = C.c_void_p()
        rc = lib.gpud_pilot_create(int(max_jobs), int(max_samples), C.byref(self._p))
        if rc != 0:
            raise GPUDError(rc, "gpud_pilot_create failed")

    def close(self):
        if self._p:
            lib.gpud_pilot_destroy(self._p)
            self._p = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, iqs, sample_rates, window: bool = True, threshold: float = 4.0):
        import torch
        keep = []
        jobs = (PilotJob * max(1, len(iqs)))()
        for i, (x, fs) in enumerate(zip(iqs, sample_rates)):
            t = x if isinstance(x, torch.Tensor) else torch.as_tensor(np.ascontiguousarray(x, np.complex64))
            t = t.to(device="cuda", dtype=torch.complex64).contiguous()
            keep.append(t)
            jobs[i] = PilotJob(t.data_ptr(), t.numel(), int(fs), 1 if window else 0, 0)
        res = (PilotResult * max(1, len(iqs)))()
        torch.cuda.synchronize()
        _check(None, lib.gpud_pilot_run(self._p, jobs, len(iqs), float(threshold), None, res))
        return [{"present": bool(r.present), "ratio": r.ratio, "best_hz": r.best_hz, "median": r.median,
                 "best_bin": r.best_bin} for r in res[: len(iqs)]]


def wfm_batch_audio(iq, sample_rate: int, offset_hz: float, bandwidth: float, deemph_us: float = 50.0):
    """Event-recording batch WFM stereo over one capture on the GPU
    (gpud_wfm_batch_audio; demodWFMStereoBatchAudio,
    recorder/wfm_batch_stereo.go:10-72).  Returns (interleaved float32 L/R at
    48 kHz, out rate, locked, demod rate)."""
    ptr, n, dev, keep = _iq_ptr(iq)
    cap = 2 * (int(n * 48000 / max(1, int(sample_rate))) + 256)
    out = np.zeros(cap, np.float32)
    res = BatchAudioResult()
    _check(None, lib.gpud_wfm_batch_audio(ptr, n, dev, int(sample_rate), float(offset_hz), float(bandwidth),
                                          float(deemph_us), out.ctypes.data, cap, C.byref(res)))
    del keep
    return out[: res.n_out].copy(), res.out_rate, bool(res.locked), res.demod_rate


def demod_audio_segment(mode: int, iq, sample_rate: int, offset_hz: float, bandwidth: float):
    """One-shot demod of a segment on the GPU (gpud_demod_audio_segment;
    demodAudioCPU, recorder/cpu_audio.go:10-75).  Returns (float32 audio,
    channels, audio rate, demod rate)."""
    ptr, n, dev, keep = _iq_ptr(iq)
    cap = 2 * n + 64
    out = np.zeros(cap, np.float32)
    res = SegmentAudioResult()
    _check(None, lib.gpud_demod_audio_segment(int(mode), ptr, n, dev, int(sample_rate), float(offset_hz),
                                              float(bandwidth), out.ctypes.data, cap, C.byref(res)))
    del keep
    return out[: res.n_out].copy(), res.channels, res.out_rate, res.demod_rate


class RDSDecoder:
    """rds.Decoder (internal/rds/rds.go:78-636) for a batch of stations on the
    device (gpud_rds_*): one Decode call per job, state per station kept on
    the device."""

    def __init__(self, max_stations: int, max_samples: int):
        self._d = C.c_void_p()
        _check(None, lib.gpud_rds_decoder_create(int(max_stations), int(max_samples), C.byref(self._d)))

    def close(self):
        if self._d:
            lib.gpud_rds_decoder_destroy(self._d)
            self._d = C.c_void_p()

    def __del__(self):
        self.close()

    def reset(self, station: int):
        _check(None, lib.gpud_rds_decoder_reset(self._d, int(station)))

    def run(self, jobs):
        """jobs: (samples, sample_rate, station) with samples a CUDA complex64
        tensor (or host data, copied to the device).  Returns one dict per job."""
        import torch
        keep, arr = [], (RDSJob * max(1, len(jobs)))()
        for k, (x, fs, st) in enumerate(jobs):
            t = x if isinstance(x, torch.Tensor) else torch.as_tensor(np.ascontiguousarray(x, np.complex64))
            t = t.to("cuda", torch.complex64).contiguous()
            keep.append(t)
            arr[k] = RDSJob(t.data_ptr() if t.numel() else None, t.numel(), int(fs), int(st), 0)
        res = (RDSResult * max(1, len(jobs)))()
        _check(None, lib.gpud_rds_decode_run(self._d, arr, len(jobs), None, res))
        return [{"groups": r.groups, "groups_total": r.groups_total, "status": r.status, "pi": r.pi,
                 "ps": r.ps.decode("ascii"), "rt": r.rt.decode("ascii")} for r in res[: len(jobs)]]

    def decode(self, samples, sample_rate: int, station: int = 0):
        return self.run([(samples, sample_rate, station)])[0]


class Spectrum:
    """Surveillance spectrum on the device (gpud_spectrum_*): fftutil.Spectrum
    and WelchPSD (internal/fft/fft.go, welch.go) in float64, power-of-two
    sizes up to 8192."""

    def __init__(self, max_fft: int = 8192, max_segments: int = 64):
        self._s = C.c_void_p()
        _check(None, lib.gpud_spectrum_create(int(max_fft), int(max_segments), C.byref(self._s)))

    def close(self):
        if self._s:
            lib.gpud_spectrum_destroy(self._s)
            self._s = C.c_void_p()

    def __del__(self):
        self.close()

    @staticmethod
    def _dev(iq):
        import torch
        t = iq if isinstance(iq, torch.Tensor) else torch.as_tensor(np.ascontiguousarray(iq, np.complex64))
        return t.to("cuda", torch.complex64).contiguous()

    def single(self, iq, hann: bool = True):
        t = self._dev(iq)
        out = np.zeros(t.numel(), np.float64)
        _check(None, lib.gpud_spectrum_single(self._s, t.data_ptr(), t.numel(), 1 if hann else 0, None,
                                              out.ctypes.data))
        return out

    def welch(self, iq, seg: int, overlap: float = 0.5, hann: bool = True):
        t = self._dev(iq)
        out = np.zeros(max(seg, t.numel()), np.float64)
        n = C.c_int()
        _check(None, lib.gpud_spectrum_welch(self._s, t.data_ptr(), t.numel(), int(seg), float(overlap),
                                             1 if hann else 0, None, out.ctypes.data, C.byref(n)))
        return out[: n.value].copy()

