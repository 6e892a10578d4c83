"""The Python mirror's ctypes structures against the C header's structs: a
probe compiled with the host C compiler prints each header struct's size and
field offsets, which must equal the ctypes layout field by field (a field
added to a header struct without its mirror, or out of order, fails here on
the CPU, before any call could read past a caller's buffer)."""
import ctypes
import os
import shutil
import subprocess

import pytest

from gpudemod import _lib as L

# header typedef -> ctypes mirror
PAIRS = {
    "gpud_channel_spec": L.ChannelSpec,
    "gpud_channel_result": L.ChannelResult,
    "gpud_autotune_entry": L.AutotuneEntry,
    "gpud_runner_stats": L.RunnerStats,
    "gpud_stage_time": L.StageTime,
    "gpud_pilot_job": L.PilotJob,
    "gpud_pilot_result": L.PilotResult,
    "gpud_batch_audio_result": L.BatchAudioResult,
    "gpud_segment_audio_result": L.SegmentAudioResult,
    "gpud_iqfile_meta": L.IQFileMeta,
    "gpud_rds_job": L.RDSJob,
    "gpud_rds_result": L.RDSResult,
}


def _probe_source():
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "gpudemod.h"', "int main(void) {"]
    for name, cls in PAIRS.items():
        lines.append(f'    printf("{name} size %zu\\n", sizeof({name}));')
        for field, _ in cls._fields_:
            lines.append(f'    printf("{name} {field} %zu\\n", offsetof({name}, {field}));')
    lines += ["    return 0;", "}"]
    return "\n".join(lines) + "\n"


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no host C compiler")
    d = tmp_path_factory.mktemp("abi")
    src, exe = d / "probe.c", d / "probe"
    src.write_text(_probe_source())
    inc = os.path.dirname(L.HEADER_PATH)
    subprocess.run([cc, "-std=c99", "-I", inc, str(src), "-o", str(exe)], check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    layout = {}
    for line in out.splitlines():
        name, field, value = line.split()
        layout[(name, field)] = int(value)
    return layout


@pytest.mark.parametrize("name", sorted(PAIRS))
def test_ctypes_mirror_matches_header(c_layout, name):
    cls = PAIRS[name]
    assert c_layout[(name, "size")] == ctypes.sizeof(cls), name
    for field, _ in cls._fields_:
        assert c_layout[(name, field)] == getattr(cls, field).offset, (name, field)

