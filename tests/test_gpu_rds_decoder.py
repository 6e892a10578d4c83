"""RDS decoding on the device (gpud_rds_*) against the oracle's restatement of
rds.Decoder.Decode (internal/rds/rds.go:78-636) on the same baseband with the
same call windows: groups per call, PI, PS and RT after every call identical,
and equal to the station's transmitted text."""
import numpy as np
import pytest

import gpudemod as G
from gpudemod import synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _rds_baseband(n_blocks=20):
    scene, st = synth.plain_wfm_scene(block=262_144)
    r = G.ChannelRunner(2_400_000, 262_144, max_channels=2)
    slot = r.admit(1, 300_000.0, 250_000.0, 300_000, 128, G.MODE_WFM_STEREO, G.CH_RDS)
    out = []
    try:
        for _ in range(n_blocks):
            r.process_block(scene.next_block().numpy())
            g = r.result(slot)
            out.append(g["rds"])
            rate = g["rds_rate"]
    finally:
        r.close()
    return out, rate, st[0]


def test_device_decoder_equals_oracle_per_call(cuda):
    blocks, rate, st = _rds_baseband()
    allb = np.concatenate(blocks)
    # three call patterns: one long window, four windows, every block alone
    windows = {0: [allb], 1: [np.concatenate(blocks[i:i + 5]) for i in range(0, 20, 5)], 2: blocks}
    dev = G.RDSDecoder(3, allb.size)
    oracles = {k: O.RDSDecoder() for k in windows}
    try:
        for call in range(max(len(v) for v in windows.values())):
            jobs = [(w[call], rate, k) for k, w in windows.items() if call < len(w)]
            got = dev.run(jobs)
            for (x, _, k), g in zip(jobs, got):
                n = oracles[k].decode(x, rate)
                pi, ps, rt = oracles[k].result()
                assert g["status"] == 0
                assert (g["groups"], g["pi"], g["ps"], g["rt"]) == (n, pi, ps, rt), (k, call)
        final = dev.run([(allb[:0], rate, 0)])[0]  # an empty call changes nothing
        assert final["pi"] == st.pi and final["ps"] == st.ps and final["groups_total"] > 10
    finally:
        dev.close()


def test_device_decoder_reset_and_short_calls(cuda):
    blocks, rate, st = _rds_baseband(8)
    x = np.concatenate(blocks)
    dev = G.RDSDecoder(2, x.size)
    ref = O.RDSDecoder()
    try:
        assert dev.decode(x[:103], rate, 1)["groups_total"] == 0  # below 104 samples: ignored
        g = dev.decode(x, rate, 1)
        assert g["groups"] == ref.decode(x, rate) and g["pi"] == ref.result()[0]
        dev.reset(1)
        again = dev.decode(x, rate, 1)
        assert again["groups"] == g["groups"] and again["groups_total"] == g["groups"]
        with pytest.raises(G.GPUDError):
            dev.run([(x, rate, 0), (x, rate, 0)])  # one job per station and run
    finally:
        dev.close()
