"""The C ABI library loads and exports every symbol include/gpudemod.h
declares (no compute calls: runs without a GPU)."""
import ctypes
import subprocess

from gpudemod._lib import LIB_PATH, header_symbols, lib


REFERENCE_SYMBOLS = [  # native/exports.cu -- all sixteen
    "gpud_stream_create", "gpud_stream_destroy", "gpud_stream_sync", "gpud_upload_fir_taps_cuda",
    "gpud_launch_freq_shift_stream_cuda", "gpud_launch_freq_shift_cuda", "gpud_launch_fm_discrim_cuda",
    "gpud_launch_fir_stream_cuda", "gpud_launch_fir_cuda", "gpud_launch_fir_v2_stream_cuda",
    "gpud_launch_decimate_stream_cuda", "gpud_launch_decimate_cuda", "gpud_launch_am_envelope_cuda",
    "gpud_launch_ssb_product_cuda", "gpud_launch_streaming_polyphase_prepare_cuda",
    "gpud_launch_streaming_polyphase_stateful_cuda",
]


def test_header_declares_reference_symbols():
    syms = header_symbols()
    for s in REFERENCE_SYMBOLS:
        assert s in syms
    assert len(set(REFERENCE_SYMBOLS)) == 16
    assert len(syms) >= 35


def test_library_exports_every_header_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [s for s in header_symbols() if s not in exported]
    assert not missing, missing
    for s in header_symbols():
        assert isinstance(getattr(lib, s), ctypes._CFuncPtr)


def test_no_non_gpud_exports():
    out = subprocess.run(["nm", "-D", "--defined-only", LIB_PATH], capture_output=True, text=True, check=True).stdout
    names = [line.split()[-1] for line in out.splitlines() if line.strip()]
    bad = [n for n in names if not n.startswith("gpud_") and not n.startswith("_")]
    assert not bad, bad[:10]


def test_host_helpers_match_reference_semantics():
    import gpudemod
    assert gpudemod.ExactIntegerDecimation(10_000_000, 312_500) == 32
    got = gpudemod.BuildPolyphaseTapsPhaseMajor(list(range(1, 8)), 3)
    assert got.tolist() == [1, 4, 7, 2, 5, 0, 3, 6, 0]
