"""Extraction-form autotuning (gpud_runner_set_autotune_table and
gpudemod.autotune): every form a class admits gives the oracle's extraction
within the parity tolerance, the table steers admission, invalid entries are
refused, and the tuner returns a valid table."""
import numpy as np
import pytest

import gpudemod as G
from gpudemod import autotune, synth
from oracle import oracle as O
from signals import rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("T,D,forms", [
    (256, 32, [G.FORM_DENSE, G.FORM_GROUP, G.FORM_WIDE]),
    (512, 400, [G.FORM_MOD, G.FORM_GROUP, G.FORM_WIDE]),
    (900, 25, [G.FORM_GROUP, G.FORM_WIDE]),
])
def test_every_form_matches_oracle(cuda, T, D, forms):
    scene, _ = synth.fm_band_scene(block=1 << 18, n_stations=8, seconds=0.2)
    xs = [scene.next_block().numpy()[: (1 << 18) - 777 * b] for b in range(2)]
    fs = 10_000_000
    if fs % (fs // D) or fs // (fs // D) != D:
        pytest.skip("inexact decimation")
    for form in forms:
        r = G.ChannelRunner(fs, 1 << 18, max_channels=2, max_taps=1024)
        r.set_autotune_table([(T, D, form, 0)])
        slot = r.admit(1, 300_000.0, 200_000.0, fs // D, T, G.MODE_IQ, G.CH_EMIT_IQ)
        assert r.channel_form(slot)[0] == form
        oc = O.OracleChannel(fs, 300_000.0, 200_000.0, fs // D, T, O.MODE_NFM, rds=False)
        try:
            for b, x in enumerate(xs):
                r.process_block(x)
                g, w = r.result(slot), oc.process(x)
                assert g["n_iq"] == w["iq"].size
                assert rel_l2(g["iq"], w["iq"]) <= 1e-5, (form, b, rel_l2(g["iq"], w["iq"]))
        finally:
            r.close()


def test_table_validation_and_tuner(cuda):
    r = G.ChannelRunner(10_000_000, 1 << 18, max_channels=2, max_taps=1024)
    try:
        with pytest.raises(G.GPUDError):
            r.set_autotune_table([(256, 32, G.FORM_MOD, 0)])  # 8 taps per arm: no modulated form
        with pytest.raises(G.GPUDError):
            r.set_autotune_table([(64, 400, G.FORM_DENSE, 0)])  # one tap per arm: no dense form
        r.set_autotune_table([])
    finally:
        r.close()
    table, report = autotune.tune(10_000_000, 1 << 18, [(256, 32), (512, 400)], channels=16, blocks=3)
    assert len(table) == 2
    for T, D, form, pg in table:
        assert (form, pg) in report[(T, D)]
        assert report[(T, D)][(form, pg)] == min(report[(T, D)].values())
    r = G.ChannelRunner(10_000_000, 1 << 18, max_channels=4, max_taps=1024)
    try:
        r.set_autotune_table(table)
        s = r.admit(1, 0.0, 10_000.0, 10_000_000 // 400, 512, G.MODE_NFM, 0)
        assert r.channel_form(s)[0] == [e for e in table if e[:2] == (512, 400)][0][2]
    finally:
        r.close()
