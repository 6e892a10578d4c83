"""ctypes binding of libgpudemod_kernels.so (include/gpudemod.h).

The library is the product; this module only declares its C ABI for Python
callers.  There is no fallback: if the shared library is missing or cannot be
loaded, importing raises.
"""
from __future__ import annotations

import ctypes as C
import os
import re

_PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(_PKG_ROOT, "libgpudemod_kernels.so")
HEADER_PATH = os.path.join(os.path.dirname(_PKG_ROOT), "include", "gpudemod.h")


class GPUDFloat2(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float)]


class ChannelSpec(C.Structure):
    """gpud_channel_spec: StreamingExtractJob (streaming_types.go:8-15) + mode."""
    _fields_ = [
        ("signal_id", C.c_int64),
        ("offset_hz", C.c_double),
        ("bandwidth", C.c_double),
        ("out_rate", C.c_int32),
        ("num_taps", C.c_int32),
        ("config_hash", C.c_uint64),
        ("mode", C.c_int32),
        ("flags", C.c_int32),
        ("demod_decim", C.c_int32),
        ("reserved", C.c_int32),
    ]


class ChannelResult(C.Structure):
    _fields_ = [
        ("signal_id", C.c_int64),
        ("rate", C.c_int32),
        ("n_iq", C.c_int32),
        ("phase_count", C.c_int32),
        ("history_len", C.c_int32),
        ("nco_phase", C.c_double),
        ("n_audio", C.c_int32),
        ("audio_channels", C.c_int32),
        ("n_rds", C.c_int32),
        ("rds_rate", C.c_int32),
        ("flags", C.c_int32),
        ("coherence", C.c_float),
        ("pilot_hz", C.c_float),
        ("err_avg", C.c_float),
        ("iq", C.POINTER(GPUDFloat2)),
        ("audio", C.POINTER(C.c_float)),
        ("rds", C.POINTER(GPUDFloat2)),
        ("pll_path", C.c_int32),
        ("pll_iters", C.c_int32),
        ("pcm", C.POINTER(C.c_int16)),
        ("n_pcm", C.c_int32),
        ("pcm_rate", C.c_int32),
        ("pcm_f32", C.POINTER(C.c_float)),
    ]


class BatchAudioResult(C.Structure):
    _fields_ = [("n_out", C.c_int32), ("out_rate", C.c_int32), ("demod_rate", C.c_int32), ("locked", C.c_int32)]


class RDSJob(C.Structure):
    _fields_ = [("samples", C.c_void_p), ("n", C.c_int32), ("sample_rate", C.c_int32), ("station", C.c_int32),
                ("pad", C.c_int32)]


class RDSResult(C.Structure):
    _fields_ = [("groups", C.c_int32), ("groups_total", C.c_int32), ("status", C.c_int32), ("pi", C.c_uint16),
                ("pad", C.c_uint16), ("ps", C.c_char * 9), ("rt", C.c_char * 65), ("pad2", C.c_char * 2)]


class AutotuneEntry(C.Structure):
    _fields_ = [("taps", C.c_int32), ("decim", C.c_int32), ("form", C.c_int32), ("group_phases", C.c_int32)]


class IQFileMeta(C.Structure):
    _fields_ = [("sample_rate", C.c_int64), ("center_hz", C.c_double), ("samples", C.c_int64)]


class SegmentAudioResult(C.Structure):
    _fields_ = [("n_out", C.c_int32), ("channels", C.c_int32), ("out_rate", C.c_int32), ("demod_rate", C.c_int32)]


class PilotJob(C.Structure):
    _fields_ = [("iq", C.c_void_p), ("n", C.c_int32), ("sample_rate", C.c_int32), ("window", C.c_int32),
                ("pad", C.c_int32)]


class PilotResult(C.Structure):
    _fields_ = [("present", C.c_int32), ("best_bin", C.c_int32), ("ratio", C.c_double), ("best_hz", C.c_double),
                ("median", C.c_double)]


class StageTime(C.Structure):
    _fields_ = [("name", C.c_char * 24), ("ms", C.c_double)]


class RunnerStats(C.Structure):
    _fields_ = [
        ("blocks", C.c_uint64),
        ("active_channels", C.c_int32),
        ("max_channels", C.c_int32),
        ("device_bytes_used", C.c_uint64),
        ("device_bytes_budget", C.c_uint64),
        ("last_block_ms", C.c_double),
        ("p50_block_ms", C.c_double),
        ("p99_block_ms", C.c_double),
        ("kernel_launches", C.c_uint64),
        ("graph_rebuilds", C.c_int32),
        ("pad", C.c_int32),
        ("last_h2d_bytes", C.c_uint64),
        ("last_d2h_bytes", C.c_uint64),
        ("ring_copy_ms", C.c_double),
        ("ring_copies", C.c_uint64),
    ]


def _declare(lib: C.CDLL) -> C.CDLL:
    P, i, d = C.c_void_p, C.c_int, C.c_double
    pi = C.POINTER(C.c_int)
    pd = C.POINTER(C.c_double)
    sig = {
        # legacy (native/exports.cu)
        "gpud_stream_create": (i, [C.POINTER(P)]),
        "gpud_stream_destroy": (i, [P]),
        "gpud_stream_sync": (i, [P]),
        "gpud_launch_freq_shift_stream_cuda": (i, [P, P, i, d, d, P]),
        "gpud_launch_freq_shift_cuda": (i, [P, P, i, d, d]),
        "gpud_launch_fm_discrim_cuda": (i, [P, P, i]),
        "gpud_upload_fir_taps_cuda": (i, [P, i]),
        "gpud_launch_fir_cuda": (i, [P, P, i, i]),
        "gpud_launch_fir_stream_cuda": (i, [P, P, i, i, P]),
        "gpud_launch_fir_v2_stream_cuda": (i, [P, P, P, i, i, P]),
        "gpud_launch_decimate_cuda": (i, [P, P, i, i]),
        "gpud_launch_decimate_stream_cuda": (i, [P, P, i, i, P]),
        "gpud_launch_am_envelope_cuda": (i, [P, P, i]),
        "gpud_launch_ssb_product_cuda": (i, [P, P, i, d, d]),
        "gpud_launch_streaming_polyphase_prepare_cuda": (
            i, [P, i, P, i, P, i, i, i, i, d, d, P, pi, pi, pd, P]),
        "gpud_launch_streaming_polyphase_stateful_cuda": (
            i, [P, i, P, P, i, i, i, P, P, i, pi, pi, pd, d, P, i, pi]),
        "gpud_launch_streaming_polyphase_stateful_noalloc_cuda": (
            i, [P, i, P, i, i, i, P, i, pi, pi, pd, d, P, i, pi]),
        # engine front end
        "gpud_lowpass_fir": (i, [d, i, i, pd, i]),
        "gpud_shift_fir_decimate_cuda": (i, [P, i, i, d, P, i, i, P, P, i, pi, P]),
        # runner
        "gpud_runner_create": (i, [i, i, i, i, C.c_uint64, C.POINTER(P)]),
        "gpud_runner_destroy": (i, [P]),
        "gpud_runner_set_autotune_table": (i, [P, C.POINTER(AutotuneEntry), i]),
        "gpud_runner_channel_form": (i, [P, i, pi, pi, pi]),
        "gpud_runner_set_channel_groups": (i, [P, i]),
        "gpud_wfm_batch_audio": (i, [P, i, i, i, d, d, d, P, i, C.POINTER(BatchAudioResult)]),
        "gpud_demod_audio_segment": (i, [i, P, i, i, i, d, d, P, i, C.POINTER(SegmentAudioResult)]),
        "gpud_iqfile_write": (i, [C.c_char_p, P, C.c_int64, C.c_int64, d]),
        "gpud_rds_decoder_create": (i, [i, i, C.POINTER(P)]),
        "gpud_spectrum_create": (i, [i, i, C.POINTER(P)]),
        "gpud_spectrum_destroy": (i, [P]),
        "gpud_spectrum_single": (i, [P, P, i, i, P, P]),
        "gpud_spectrum_welch": (i, [P, P, C.c_int64, i, d, i, P, P, pi]),
        "gpud_rds_decoder_destroy": (i, [P]),
        "gpud_rds_decoder_reset": (i, [P, i]),
        "gpud_rds_decode_run": (i, [P, C.POINTER(RDSJob), i, P, C.POINTER(RDSResult)]),
        "gpud_iqfile_open": (i, [C.c_char_p, C.POINTER(P), C.POINTER(IQFileMeta)]),
        "gpud_iqfile_close": (None, [P]),
        "gpud_iqfile_read": (i, [P, P, C.c_int64, i, P]),
        "gpud_iqfile_seek": (i, [P, C.c_int64]),
        "gpud_iqfile_tell": (C.c_int64, [P]),
        "gpud_runner_admit": (i, [P, C.POINTER(ChannelSpec), pi]),
        "gpud_runner_retire": (i, [P, i]),
        "gpud_runner_update": (i, [P, i, d, d]),
        "gpud_runner_set_schedule": (i, [P, i]),
        "gpud_runner_channel_footprint": (i, [P, C.POINTER(ChannelSpec), C.POINTER(C.c_uint64)]),
        "gpud_runner_process_block": (i, [P, P, i, i]),
        "gpud_runner_submit": (i, [P, P, i, i, C.POINTER(C.c_uint64)]),
        "gpud_runner_wait": (i, [P, C.c_uint64, i]),
        "gpud_runner_result": (i, [P, i, C.POINTER(ChannelResult)]),
        "gpud_runner_stats_get": (i, [P, C.POINTER(RunnerStats)]),
        "gpud_runner_reset_stats": (i, [P]),
        "gpud_runner_stream": (i, [P, C.POINTER(P)]),
        "gpud_runner_last_error": (C.c_char_p, [P]),
        "gpud_runner_snapshot": (i, [P, i, P, C.POINTER(C.c_uint64)]),
        "gpud_runner_restore": (i, [P, i, P, C.c_uint64]),
        "gpud_runner_streaming_extract": (i, [P, P, i, C.POINTER(ChannelSpec), i, C.POINTER(ChannelResult), P, i]),
        "gpud_runner_reset_signal": (i, [P, C.c_int64]),
        "gpud_runner_set_host_outputs": (i, [P, i]),
        "gpud_runner_set_profiling": (i, [P, i]),
        "gpud_runner_set_pll_solver": (i, [P, i]),
        "gpud_runner_stage_times": (i, [P, C.POINTER(StageTime), i, pi]),
        "gpud_runner_reset_all_signals": (i, [P]),
        "gpud_streaming_config_hash": (C.c_uint64, [C.c_int64, i, i, i]),
        "gpud_kernel_launch_count": (C.c_uint64, []),
        "gpud_pilot_create": (i, [i, i, C.POINTER(P)]),
        "gpud_pilot_destroy": (i, [P]),
        "gpud_pilot_run": (i, [P, C.POINTER(PilotJob), i, d, P, C.POINTER(PilotResult)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def header_symbols(path: str = HEADER_PATH) -> list[str]:
    """Every function the public header declares."""
    txt = open(path).read()
    return sorted(set(re.findall(r"GPUD_CALL\s+(gpud_\w+)\s*\(", txt)))


def load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `make -C argus-sdr_b200` "
                          f"(or __graft_entry__.build()); there is no non-CUDA fallback")
    return _declare(C.CDLL(LIB_PATH))


lib = load()
