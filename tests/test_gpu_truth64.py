"""Error against a float64 truth, per output: the GPU chain and the
reference-precision restatement (the oracle), each against the same chain
evaluated entirely in float64 (oracle/truth64.py).  Both must stay within the
parity tolerance (relative L2 <= 1e-5 per output stream); the GPU's error
is reported next to the oracle's.  With GPUD_PARITY_REPORT set to a path the
table is written there as JSON."""
import json
import os

import numpy as np
import pytest

import gpudemod as G
from gpudemod import synth
from oracle import oracle as O
from oracle import truth64 as T64

pytestmark = pytest.mark.gpu

TOL = 1e-5
_REPORT = {}


def _err(a, b):
    a = np.concatenate([np.asarray(x, np.complex128).ravel() for x in a]) if a else np.zeros(0)
    b = np.concatenate([np.asarray(x, np.complex128).ravel() for x in b]) if b else np.zeros(0)
    assert a.size == b.size
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)) if b.size else 0.0


def _run(case, fs, block, blocks, spec, rds):
    sid, off, bw, rate, taps, mode, flags = spec
    gr = G.ChannelRunner(fs, block, max_channels=2, max_taps=1024)
    slot = gr.admit(sid, off, bw, rate, taps, mode, flags | G.CH_EMIT_IQ)
    oc = O.OracleChannel(fs, off, bw, rate, taps, mode, rds=rds)
    tc = T64.Truth64Channel(fs, off, bw, rate, taps, mode, rds=rds)
    outs = {k: ([], [], []) for k in ("iq", "audio_L", "audio_R", "audio", "rds")}
    try:
        for x in blocks:
            gr.process_block(x)
            g, o, t = gr.result(slot), oc.process(x), tc.process(x)
            assert g["locked"] == o["locked"] == t["locked"]
            assert g["stereo"] == o["stereo"] == t["stereo"]
            for src, res in zip(range(3), (g, o, t)):
                outs["iq"][src].append(res["iq"])
                outs["rds"][src].append(res["rds"])
                if mode == G.MODE_WFM_STEREO:
                    outs["audio_L"][src].append(res["audio"][0::2])
                    outs["audio_R"][src].append(res["audio"][1::2])
                else:
                    outs["audio"][src].append(res["audio"])
    finally:
        gr.close()
    row = {}
    for name, (gg, oo, tt) in outs.items():
        if not tt or sum(np.asarray(v).size for v in tt) == 0:
            continue
        row[name] = {"gpu_vs_f64": _err(gg, tt), "oracle_vs_f64": _err(oo, tt), "gpu_vs_oracle": _err(gg, oo)}
        assert row[name]["gpu_vs_f64"] <= TOL, (case, name, row[name])
        assert row[name]["oracle_vs_f64"] <= TOL, (case, name, row[name])
    _REPORT[case] = row


def test_plain_wfm_stereo_rds_vs_f64(cuda):
    scene, _ = synth.plain_wfm_scene(block=262_144)
    blocks = [scene.next_block().numpy() for _ in range(8)]
    _run("plain WFM stereo + RDS (2.4 MS/s, 128 taps, D 8)", 2_400_000, 262_144, blocks,
         (1, 300_000.0, 250_000.0, 300_000, 128, G.MODE_WFM_STEREO, G.CH_RDS), True)


def test_fm_band_channel_vs_f64(cuda):
    scene, st = synth.fm_band_scene(device="cuda", block=1 << 20, n_stations=40, seconds=5.0)
    blocks = [scene.next_block().cpu().numpy() for _ in range(5)]
    _run("FM band WFM stereo + RDS (10 MS/s, 256 taps, D 32)", 10_000_000, 1 << 20, blocks,
         (1, st[7].offset_hz, 250_000.0, 312_500, 256, G.MODE_WFM_STEREO, G.CH_RDS), True)


@pytest.mark.parametrize("kind", ["NFM", "AM", "USB", "LSB", "CW"])
def test_mixed_mode_channel_vs_f64(cuda, kind):
    scene, chans = synth.mixed_scene(device="cuda", block=1 << 20)
    blocks = [scene.next_block().cpu().numpy() for _ in range(3)]
    off = next(o for k, o in chans if k == kind)
    rate, taps, bw = synth.MODE_TABLE[kind]
    mode = {"NFM": G.MODE_NFM, "AM": G.MODE_AM, "USB": G.MODE_USB, "LSB": G.MODE_LSB, "CW": G.MODE_CW}[kind]
    _run(f"mixed batch {kind} (10 MS/s, {taps} taps, D {10_000_000 // rate})", 10_000_000, 1 << 20, blocks,
         (1, off, bw, rate, taps, mode, 0), False)


def test_zz_write_parity_report():
    path = os.environ.get("GPUD_PARITY_REPORT")
    if path and _REPORT:
        with open(path, "w") as f:
            json.dump(_REPORT, f, indent=1)
