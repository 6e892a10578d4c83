"""The full per-channel chain on the GPU runner (extract -> demod -> WFM
multiplex -> RDS baseband) against the CPU oracle chain, block by block."""
import numpy as np
import pytest

import gpudemod as G
from gpudemod import synth
from oracle import oracle as O
from signals import max_abs, rel_l2

pytestmark = pytest.mark.gpu

AUDIO_TOL = 1e-5   # relative L2 per block (the parity tolerance)
RDS_TOL = 1e-5


def _scene_blocks(n_blocks, block=262_144, seed=synth.CONFIG_SEEDS[0]):
    scene, st = synth.plain_wfm_scene(block=block, seed=seed)
    return [scene.next_block().numpy() for _ in range(n_blocks)], st


def _compare_block(g, w, ctx):
    assert g["n_iq"] == w["iq"].size, ctx
    assert g["audio"].size == w["audio"].size, ctx
    assert g["rds"].size == w["rds"].size, ctx
    if w["audio"].size:
        assert rel_l2(g["audio"], w["audio"]) <= AUDIO_TOL, (ctx, rel_l2(g["audio"], w["audio"]))
    if w["rds"].size:
        assert rel_l2(g["rds"], w["rds"]) <= RDS_TOL, (ctx, rel_l2(g["rds"], w["rds"]))
    assert g["locked"] == w["locked"], ctx
    assert g["stereo"] == w["stereo"], ctx


def test_wfm_stereo_rds_chain_matches_oracle(cuda):
    # 20 blocks = 2.2 s: more than one full RDS group cycle (20 groups, 1.75 s)
    blocks, st = _scene_blocks(20)
    fs, out = 2_400_000, 300_000
    runner = G.ChannelRunner(fs, 262_144, max_channels=4)
    slot = runner.admit(1, 300_000.0, 250_000.0, out, 128, G.MODE_WFM_STEREO, G.CH_RDS | G.CH_EMIT_IQ)
    ref = O.OracleChannel(fs, 300_000.0, 250_000.0, out, 128, O.MODE_WFM_STEREO, rds=True)
    g_rds, w_rds = [], []
    try:
        for b, x in enumerate(blocks):
            runner.process_block(x)
            g = runner.result(slot)
            w = ref.process(x)
            assert rel_l2(g["iq"], w["iq"]) <= 1e-5
            _compare_block(g, w, b)
            c, f, e = ref.margins()
            assert abs(g["coherence"] - c) <= 1e-4 * max(1, c)
            assert abs(g["pilot_hz"] - f) <= 1e-2
            g_rds.append(g["rds"])
            w_rds.append(w["rds"])
        # RDS groups decoded from the GPU baseband == from the oracle baseband
        dg, dw = O.RDSDecoder(), O.RDSDecoder()
        ng = dg.decode(np.concatenate(g_rds), 20_000)
        nw = dw.decode(np.concatenate(w_rds), 20_000)
        assert ng == nw and ng > 0
        assert dg.result() == dw.result()
        assert dg.result()[0] == st[0].pi and dg.result()[1] == st[0].ps
        assert runner.result(slot)["stereo"]
    finally:
        runner.close()


@pytest.mark.parametrize("mode,out_rate,taps,bw,offset", [
    (G.MODE_NFM, 25_000, 512, 12_500, -400_000.0),
    (G.MODE_AM, 25_000, 384, 10_000, 150_000.0),
    (G.MODE_USB, 12_500, 256, 3_000, 612_345.0),
    (G.MODE_LSB, 12_500, 256, 3_000, -512_345.0),
    (G.MODE_CW, 5_000, 128, 500, 1_000_000.0),
    (G.MODE_WFM, 312_500, 256, 250_000, -2_000_000.0),
])
def test_narrow_modes_match_oracle(cuda, mode, out_rate, taps, bw, offset):
    fs, block = 10_000_000, 200_000
    rng = np.random.default_rng(mode)
    runner = G.ChannelRunner(fs, block, max_channels=2)
    slot = runner.admit(9, offset, bw, out_rate, taps, mode, G.CH_EMIT_IQ)
    ref = O.OracleChannel(fs, offset, bw, out_rate, taps, mode, rds=False)
    try:
        for b in range(4):
            n = block - 17 * b
            t = np.arange(b * block, b * block + n)
            # a tone carrier; for AM a 1 kHz tone at 50 % modulation, so the
            # demodulated audio is not a vanishing difference of two envelopes
            env = 1.0 + (0.5 * np.sin(2 * np.pi * 1000 * t / fs) if mode == G.MODE_AM else 0.0)
            x = (0.3 * (rng.standard_normal(n) + 1j * rng.standard_normal(n))
                 + env * np.exp(2j * np.pi * (offset + 1234.5) * t / fs)).astype(np.complex64)
            runner.process_block(x)
            g = runner.result(slot)
            w = ref.process(x)
            assert rel_l2(g["iq"], w["iq"]) <= 1e-5
            assert g["audio"].size == w["audio"].size
            assert rel_l2(g["audio"], w["audio"]) <= AUDIO_TOL, rel_l2(g["audio"], w["audio"])
            assert g["phase_count"] == ref.state()[1] and g["history_len"] == ref.state()[2]
    finally:
        runner.close()


def _mixed_runner(fs, block, schedule=G.SCHED_BATCHED):
    r = G.ChannelRunner(fs, block, max_channels=16)
    r.set_schedule(schedule)
    specs = [
        (1, 300_000.0, 250_000.0, 300_000, 128, G.MODE_WFM_STEREO, G.CH_RDS | G.CH_EMIT_IQ),
        (2, -450_000.0, 12_500.0, 25_000, 512, G.MODE_NFM, 0),
        (3, 700_000.0, 10_000.0, 25_000, 384, G.MODE_AM, 0),
        (4, -900_000.0, 3_000.0, 12_500, 256, G.MODE_USB, 0),
        (5, 100_000.0, 500.0, 5_000, 128, G.MODE_CW, 0),
    ]
    slots = [r.admit(*s) for s in specs]
    return r, slots, specs


def test_batched_equals_plain_schedule(cuda):
    blocks, _ = _scene_blocks(3)
    fs = 2_400_000
    rb, sb, _ = _mixed_runner(fs, 262_144)
    rp, sp, _ = _mixed_runner(fs, 262_144, G.SCHED_PLAIN)
    try:
        for x in blocks:
            rb.process_block(x)
            rp.process_block(x)
            for a, b in zip(sb, sp):
                ga, gb = rb.result(a), rp.result(b)
                assert np.array_equal(ga["audio"], gb["audio"])
                assert np.array_equal(ga["rds"], gb["rds"])
                assert np.array_equal(ga["iq"], gb["iq"])
                assert ga["stereo"] == gb["stereo"]
    finally:
        rb.close()
        rp.close()


def test_channel_alone_equals_in_mix(cuda):
    """Serving invariant: a channel's output is identical alone and in a mix."""
    blocks, _ = _scene_blocks(3)
    fs = 2_400_000
    mix, slots, specs = _mixed_runner(fs, 262_144)
    try:
        for k, spec in enumerate(specs):
            alone = G.ChannelRunner(fs, 262_144, max_channels=2)
            s = alone.admit(*spec)
            outs_alone = []
            for x in blocks:
                alone.process_block(x)
                outs_alone.append(alone.result(s))
            alone.close()
            if k == 0:
                outs_mix = [[] for _ in specs]
                for x in blocks:
                    mix.process_block(x)
                    for j, sl in enumerate(slots):
                        outs_mix[j].append(mix.result(sl))
            for a, m in zip(outs_alone, outs_mix[k]):
                assert np.array_equal(a["audio"], m["audio"])
                assert np.array_equal(a["rds"], m["rds"])
                assert a["stereo"] == m["stereo"]
    finally:
        mix.close()


def test_snapshot_restore_continues_exactly(cuda):
    blocks, _ = _scene_blocks(4)
    fs = 2_400_000
    spec = (1, 300_000.0, 250_000.0, 300_000, 128, G.MODE_WFM_STEREO, G.CH_RDS)
    ra = G.ChannelRunner(fs, 262_144, max_channels=2)
    rb = G.ChannelRunner(fs, 262_144, max_channels=2)
    sa = ra.admit(*spec)
    try:
        for x in blocks[:2]:
            ra.process_block(x)
        blob = ra.snapshot(sa)
        sb = rb.admit(*spec)
        rb.restore(sb, blob)
        for x in blocks[2:]:
            ra.process_block(x)
            rb.process_block(x)
            a, b = ra.result(sa), rb.result(sb)
            assert np.array_equal(a["audio"], b["audio"])
            assert np.array_equal(a["rds"], b["rds"])
    finally:
        ra.close()
        rb.close()


def test_admission_by_device_memory_budget(cuda):
    fs, block = 10_000_000, 262_144
    probe = G.ChannelRunner(fs, block, max_channels=8)
    fp = probe.footprint(312_500, G.MODE_WFM_STEREO, G.CH_RDS, 256)
    base = probe.stats()["device_bytes_used"]
    probe.close()
    r = G.ChannelRunner(fs, block, max_channels=8, device_mem_budget=base + 3 * fp + fp // 2)
    try:
        for i in range(3):
            r.admit(i, 100_000.0 * i, 250_000.0, 312_500, 256, G.MODE_WFM_STEREO, G.CH_RDS)
        with pytest.raises(G.GPUDError) as ei:
            r.admit(9, 0.0, 250_000.0, 312_500, 256, G.MODE_WFM_STEREO, G.CH_RDS)
        assert ei.value.code == G.E_BUDGET
        r.retire(0)
        r.admit(9, 0.0, 250_000.0, 312_500, 256, G.MODE_WFM_STEREO, G.CH_RDS)
    finally:
        r.close()


def test_parallel_pll_equals_serial_pll(cuda):
    """The Newton/scan PLL solver reproduces the serial loop (same recurrence)
    and takes over once the loop is locked."""
    blocks, _ = _scene_blocks(8)
    fs = 2_400_000
    spec = (1, 300_000.0, 250_000.0, 300_000, 128, G.MODE_WFM_STEREO, G.CH_RDS)
    rp = G.ChannelRunner(fs, 262_144, max_channels=2)
    rs = G.ChannelRunner(fs, 262_144, max_channels=2)
    rs.set_pll_solver(False)
    sp, ss = rp.admit(*spec), rs.admit(*spec)
    paths = []
    try:
        for x in blocks:
            rp.process_block(x)
            rs.process_block(x)
            a, b = rp.result(sp), rs.result(ss)
            paths.append(a["pll_path"])
            assert b["pll_path"] == 2
            assert rel_l2(a["audio"], b["audio"]) <= 1e-6, rel_l2(a["audio"], b["audio"])
            assert a["locked"] == b["locked"] and a["stereo"] == b["stereo"]
            assert abs(a["coherence"] - b["coherence"]) <= 1e-5
        # acquisition from zero I/Q included: every block by the parallel solver
        assert all(p == 1 for p in paths), paths
    finally:
        rp.close()
        rs.close()


def test_parallel_pll_fallback_and_clusters(cuda):
    """Several stereo channels (split over thread-block clusters), some without
    a pilot: blocks that do not converge fall back to the serial loop; every
    block matches the serial-only solver."""
    blocks, _ = _scene_blocks(6)
    fs = 2_400_000
    specs = [(1, 300_000.0, 250_000.0, 300_000, 128, G.MODE_WFM_STEREO, G.CH_RDS),
             (2, -500_000.0, 250_000.0, 300_000, 128, G.MODE_WFM_STEREO, G.CH_RDS),
             (3, 800_000.0, 250_000.0, 300_000, 128, G.MODE_WFM_STEREO, 0)]
    rp = G.ChannelRunner(fs, 262_144, max_channels=4)
    rs = G.ChannelRunner(fs, 262_144, max_channels=4)
    rc = G.ChannelRunner(fs, 262_144, max_channels=4)
    rs.set_pll_solver(False)
    rc.set_pll_solver(True, max_iters=3)  # too few for acquisition: those blocks fall back
    sp = [rp.admit(*s) for s in specs]
    ss = [rs.admit(*s) for s in specs]
    sc = [rc.admit(*s) for s in specs]
    paths, cpaths = set(), set()
    try:
        for x in blocks:
            for r in (rp, rs, rc):
                r.process_block(x)
            for a_slot, b_slot, c_slot in zip(sp, ss, sc):
                a, b, c = rp.result(a_slot), rs.result(b_slot), rc.result(c_slot)
                paths.add(a["pll_path"])
                cpaths.add(c["pll_path"])
                for o in (a, c):
                    assert rel_l2(o["audio"], b["audio"]) <= 1e-6, rel_l2(o["audio"], b["audio"])
                    assert o["locked"] == b["locked"] and o["stereo"] == b["stereo"]
        assert 1 in paths
        assert 2 in cpaths, cpaths
    finally:
        rp.close()
        rs.close()
        rc.close()



@pytest.mark.parametrize("depth", [2, 3])
def test_pipelined_submit_equals_sequential(cuda, depth):
    """Two or three blocks in flight (block k+1's front half overlapping block k's PLL
    and stereo output), with drift updates, retires and admissions made while
    a block is in flight: every output is bit-identical to the one block at a
    time runner given the same calls at the same block boundaries."""
    blocks, _ = _scene_blocks(8)
    fs = 2_400_000
    rs, ss, _ = _mixed_runner(fs, 262_144)
    rp, sp, _ = _mixed_runner(fs, 262_144)
    late = [(7, -200_000.0, 250_000.0, 300_000, 128, G.MODE_WFM, G.CH_RDS),
            (8, 500_000.0, 250_000.0, 300_000, 128, G.MODE_WFM_STEREO, G.CH_RDS | G.CH_EMIT_IQ)]
    keys = ("audio", "rds", "iq", "n_iq", "phase_count", "history_len", "nco_phase", "stereo", "locked",
            "coherence", "pilot_hz", "err_avg", "pll_path")

    def calls(r, live, k):
        # control calls made after block k (on the pipelined runner: while
        # block k is in flight)
        if k == 2:
            r.update(live[2], -451_000.0, 12_500.0)      # NCO drift
            r.update(live[4], -900_000.0, 2_400.0)       # taps rebuilt
        if k == 3:
            r.retire(live.pop(5))                        # CW
        if k == 4:
            live[7] = r.admit(*late[0])
        if k == 5:
            r.retire(live.pop(3))                        # AM
            live[8] = r.admit(*late[1])

    def collect(r, live):
        return {sid: r.result(slot) for sid, slot in live.items()}

    live_s = {sid: slot for sid, slot in zip(range(1, 6), ss)}
    live_p = {sid: slot for sid, slot in zip(range(1, 6), sp)}
    seq, pipe = [], []
    try:
        for k, x in enumerate(blocks):
            rs.process_block(x)
            seq.append(collect(rs, live_s))
            calls(rs, live_s, k)
        tickets = []
        for k, x in enumerate(blocks):
            tickets.append(rp.submit(x))
            if k >= depth - 1:
                rp.wait(tickets[k - depth + 1])
                pipe.append(collect(rp, live_p))
            calls(rp, live_p, k)
        for k in range(len(blocks) - depth + 1, len(blocks)):
            rp.wait(tickets[k])
            pipe.append(collect(rp, live_p))
        assert len(seq) == len(pipe) == len(blocks)
        for k, (a, b) in enumerate(zip(seq, pipe)):
            # block k's results are read after the calls made while it was in
            # flight: a channel retired then has none, one admitted then did
            # not take part in block k
            common = a.keys() & b.keys()
            assert len(common) >= len(a) - 1, k
            for sid in b.keys() - a.keys():
                assert b[sid]["n_iq"] == 0 and b[sid]["audio"].size == 0, (k, sid)
            for sid in common:
                for key in keys:
                    va, vb = a[sid][key], b[sid][key]
                    same = np.array_equal(va, vb) if isinstance(va, np.ndarray) else va == vb
                    assert same, (k, sid, key)
        st = rp.stats()
        assert st["blocks"] == len(blocks) and st["p99_block_ms"] > 0
    finally:
        rs.close()
        rp.close()
