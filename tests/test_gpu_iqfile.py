"""A snapshot replayed from an SDRIQ001 file straight into device memory
(the mapped file page-locked, one copy per block and wrap) runs through the
runner exactly as the same blocks from host memory."""
import numpy as np
import pytest

import gpudemod as G
from gpudemod import iqfile, synth

pytestmark = pytest.mark.gpu


def test_replay_into_runner_equals_host_blocks(cuda, tmp_path):
    scene, _ = synth.plain_wfm_scene(block=65_536)
    x = np.concatenate([scene.next_block().numpy() for _ in range(5)])
    p = tmp_path / "fm.cf32"
    iqfile.write(p, x, 2_400_000, 100.0e6)
    src = iqfile.Source(p, paced=False)
    assert src.meta.SampleRate == 2_400_000
    spec = (1, 300_000.0, 250_000.0, 300_000, 128, G.MODE_WFM_STEREO, G.CH_RDS | G.CH_AUDIO48K)
    ra = G.ChannelRunner(2_400_000, 100_000, max_channels=2)
    rb = G.ChannelRunner(2_400_000, 100_000, max_channels=2)
    sa, sb = ra.admit(*spec), rb.admit(*spec)
    try:
        pos = 0
        for k, n in enumerate([100_000, 77_777, 100_000, 50_000]):  # the last read wraps
            dev = src.read_iq(n, device="cuda")
            host = np.concatenate([x, x])[pos:pos + n]
            pos = (pos + n) % x.size
            assert np.array_equal(dev.cpu().numpy(), host)
            ra.process_block(dev)
            rb.process_block(host)
            a, b = ra.result(sa), rb.result(sb)
            for key in ("pcm", "rds"):
                assert np.array_equal(a[key], b[key]), (k, key)
    finally:
        ra.close()
        rb.close()
        src.close()
