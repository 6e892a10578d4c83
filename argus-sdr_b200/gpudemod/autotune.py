"""Extraction-form autotuner: for each channel class (applied tap count T,
decimation D) it times every form the geometry admits -- dense tiles, phase
groups at two group sizes, the modulated short-arm form, the warp-per-output
form -- on a scratch runner filled with channels of that class, and keeps the
fastest.  The result is a table for ChannelRunner.set_autotune_table; a
channel's form then depends on its class alone, so (with channel groups off)
outputs stay identical alone and in any mix under one table.

Timing: the runner's per-stage CUDA events around the extraction launches of
steady blocks (the first block of each trial is a warm-up).  Trials run with
the runner's default channel groups, so the dense candidate of a class
measures the tensor-core group kernel that a deployment with four or more
channels of the class would run (and the dense kernel for the first 256
outputs, on the side stream, inside the group's interval)."""
from __future__ import annotations

import statistics

import numpy as np

from . import FORM_DENSE, FORM_GROUP, FORM_MOD, FORM_WIDE, GPUDError, MODE_IQ, ChannelRunner

# every extraction stage, the channel-group taps packing included (a repack
# runs only when the group or a member's taps change, so a steady trial
# mostly sees the group kernel itself)
_EXTRACT_STAGES = ("extract", "gemm_pack")


def _candidates(T: int, D: int):
    L = -(-T // D)
    out = [(FORM_WIDE, 0), (FORM_GROUP, 0)]
    P = min(T, D)
    if P >= 16:
        out.append((FORM_GROUP, max(1, P // 4)))
    if 2 <= L <= 16:
        out.append((FORM_DENSE, 0))
    if L <= 4:
        out.append((FORM_MOD, 0))
    return out


def _trial(fs, block, T, D, form, pg, channels, blocks, x):
    r = ChannelRunner(fs, block, max_channels=channels, max_taps=max(T, 64))
    try:
        r.set_autotune_table([(T, D, form, pg)])
        for i in range(channels):
            r.admit(i, (i - channels / 2) * 1e3, 10_000.0, fs // D, T, MODE_IQ, 0)
        r.set_host_outputs(False)
        r.set_profiling(True)
        times = []
        for b in range(blocks):
            r.process_block(x)
            if b:
                times.append(sum(ms for name, ms in r.stage_times() if name.startswith(_EXTRACT_STAGES)))
        return statistics.median(times)
    finally:
        r.close()


def tune(fs: int, block: int, classes, channels: int = 32, blocks: int = 4, seed: int = 1):
    """classes: iterable of (T, D).  Returns (table, report): table entries
    (T, D, form, group_phases) of the fastest form per class, report the
    per-candidate times in ms."""
    import torch
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    x = (torch.randn(block, 2, device="cuda", generator=g) * 0.1).contiguous().view(torch.complex64).reshape(block)
    table, report = [], {}
    for T, D in classes:
        best, times = None, {}
        for form, pg in _candidates(int(T), int(D)):
            try:
                ms = _trial(fs, block, int(T), int(D), form, pg, channels, blocks, x)
            except GPUDError:
                continue  # the geometry does not admit this form
            times[(form, pg)] = ms
            if best is None or ms < times[best]:
                best = (form, pg)
        report[(T, D)] = times
        if best is not None:
            table.append((int(T), int(D), best[0], best[1]))
    return table, report
