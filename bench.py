"""Benchmark: aggregate channel-MS/s of the gpudemod runner on one B200.

Workload (default): the FM-band batch -- 10 MS/s cf32 IQ in blocks of 2^20
samples, 40 WFM stations on a 200 kHz grid (10-40 dB SNR), each extracted with
a 256-tap FIR decimating by 32 to 312.5 kS/s, FM-discriminated, stereo-decoded
(19 kHz pilot PLL, 38 kHz L-R) and RDS-baseband-extracted, all channels in one
launch sequence per block.  A step is one block through every channel.

  value      channel-MS/s with the IQ blocks already in HBM (>= 64 consecutive
             seeded blocks of one continuous stream, >= 512 MiB > L2), outputs
             left on the device
  e2e        the same through the public C ABI from pinned host memory: H2D of
             the block, all kernels, D2H of audio + RDS + results, every step
  plain      the per-signal plain runner (one channel at a time, H2D/D2H per
             channel) on the same GPU and workload
  roofline   the dominant kernel, measured live from CUDA events between the
             runner's launches over the timed region
  cpu_baseline  the oracle (C restatement of the reference's Go CPU path) on a
             bounded sample, all host threads

`--impl reference` times the reference CPU path (the oracle port; the
reference is Go and no Go toolchain exists on the box) on the same workload.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "argus-sdr_b200"))

import numpy as np  # noqa: E402

FS = 10_000_000
BLOCK = 1 << 20
N_CH = 40
TAPS = 256
OUT_RATE = 312_500
BW = 250_000.0
N_BLOCKS = 64
METRIC = "aggregate channel-MS/s on 1 B200 (serving vs plain runner); p99 block latency"
WORKLOAD = ("FM band batch: 10 MS/s cf32, 2^20-sample blocks, 40 WFM stations on a 200 kHz grid "
            "(10-40 dB SNR), 256-tap FIR, decimate by 32 to 312.5 kS/s, FM discriminator, stereo "
            "decode with 19 kHz pilot PLL, RDS baseband")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--plain-steps", type=int, default=3)
    ap.add_argument("--cpu-blocks", type=int, default=2, help="cpu_baseline sample: blocks of 2^20 per channel")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--profile-only", action="store_true", help="short run for ncu (no baselines)")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# distributed plumbing: gpudemod.dist (one process per GPU, channels sharded,
# no data-path collective; a barrier and a max-reduction of timings only)
# ---------------------------------------------------------------------------
def dist_setup(n_gpus):
    from gpudemod import dist as D
    return D.init("nccl")


def barrier(world):
    from gpudemod import dist as D
    D.barrier(world)


def max_over_ranks(world, v: float) -> float:
    from gpudemod import dist as D
    return D.max_over_ranks(world, v, device="cuda")


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------
def make_scene(device, rank=0, n_blocks=N_BLOCKS):
    import torch

    from gpudemod import synth
    scene, stations = synth.fm_band_scene(device=device, block=BLOCK, n_stations=N_CH,
                                          seconds=n_blocks * BLOCK / FS + 1, seed=synth.CONFIG_SEEDS[1] + rank)
    blocks = torch.empty((n_blocks, BLOCK), dtype=torch.complex64, device=device)
    for b in range(n_blocks):
        blocks[b] = scene.next_block()
    return blocks, stations


def admit_all(runner, stations):
    import gpudemod as G
    return [runner.admit(i, st.offset_hz, BW, OUT_RATE, TAPS, G.MODE_WFM_STEREO, G.CH_RDS)
            for i, st in enumerate(stations)]


def algorithmic_work():
    """Per block, per channel (the definitions the reference workload implies):
    extraction 4*T*n_out + min(6*n_in, 4*T*n_out) flop; composite demod
    (3 stereo FIRs + L-R FIR of 101 taps at 2 flop/tap + PLL ~36 + discriminator 6)
    per composite sample; RDS 4*101 per RDS output + 2 per composite sample.
    Bytes: the block read once + outputs + per-channel state."""
    n_out = BLOCK // (FS // OUT_RATE)
    dr = OUT_RATE // 19000
    n_rds = n_out // dr
    f_extract = 4 * TAPS * n_out + min(6 * BLOCK, 4 * TAPS * n_out)
    f_wfm_fir = 3 * 2 * 101 * n_out
    f_wfm_out = 2 * 101 * n_out
    f_pll = 36 * n_out
    f_demod = 6 * n_out
    f_rds = 404 * n_rds + 2 * n_out
    state_b = 4 * TAPS + 16 * (TAPS - 1)
    return {
        "extract": {"flop": f_extract * N_CH, "bytes": 8 * BLOCK + N_CH * (8 * n_out + state_b)},
        "wfm_fir": {"flop": f_wfm_fir * N_CH, "bytes": N_CH * n_out * 4 * 4},
        "wfm_out": {"flop": f_wfm_out * N_CH, "bytes": N_CH * n_out * (4 * 2 + 8)},
        "pll": {"flop": f_pll * N_CH, "bytes": N_CH * n_out * 12},
        "demod": {"flop": f_demod * N_CH, "bytes": N_CH * n_out * 12},
        "rds": {"flop": f_rds * N_CH, "bytes": N_CH * (n_out * 4 + n_rds * 8)},
        "per_block_flop": (f_extract + f_wfm_fir + f_wfm_out + f_pll + f_demod + f_rds) * N_CH,
    }


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def fp32_peak_tflops():
    """cuBLAS SGEMM (TF32 off) 8192^3 as the measured FP32 FMA peak on this GPU."""
    import torch
    torch.backends.cuda.matmul.allow_tf32 = False
    a = torch.randn(8192, 8192, device="cuda")
    b = torch.randn(8192, 8192, device="cuda")
    for _ in range(2):
        a @ b
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = 1e9
    for _ in range(5):
        e0.record()
        a @ b
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    return 2 * 8192 ** 3 / (best * 1e-3) / 1e12


# ---------------------------------------------------------------------------
# CPU path (oracle restatement of the reference's Go CPU code)
# ---------------------------------------------------------------------------
def cpu_run(blocks_np, stations, n_blocks, threads):
    from oracle import oracle as O
    chans = [O.OracleChannel(FS, st.offset_hz, BW, OUT_RATE, TAPS, O.MODE_WFM_STEREO, rds=True) for st in stations]

    def work(c):
        for b in range(n_blocks):
            c.process(blocks_np[b % len(blocks_np)])

    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(max_workers=threads) as ex:
        list(ex.map(work, chans))
    dt = time.perf_counter() - t0
    return len(chans) * n_blocks * BLOCK / dt / 1e6, dt


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


# ---------------------------------------------------------------------------
def run_reference(args):
    world, rank, local = dist_setup(args.gpus)
    if rank != 0:
        barrier(world)
        return
    import torch
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    nb = 2
    blocks, stations = make_scene(dev, 0, n_blocks=nb)
    blocks_np = [b.cpu().numpy() for b in blocks]
    threads = host_threads()
    # each step: every channel processes one 2^18-sample chunk (a bounded sample
    # of the 2^20 block) through the full chain, state carried across steps
    from oracle import oracle as O
    chans = [O.OracleChannel(FS, st.offset_hz, BW, OUT_RATE, TAPS, O.MODE_WFM_STEREO, rds=True) for st in stations]
    chunk = 1 << 18
    pos = [0]

    def step():
        b = pos[0]
        src = blocks_np[(b * chunk // BLOCK) % nb]
        off = (b * chunk) % BLOCK
        x = src[off:off + chunk]
        with cf.ThreadPoolExecutor(max_workers=threads) as ex:
            list(ex.map(lambda c: c.process(x), chans))
        pos[0] += 1

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = time.perf_counter() - t0
    v = N_CH * chunk * args.steps / dt / 1e6
    line = {"metric": METRIC, "value": v, "unit": "channel-MS/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64", "data": "synthetic (seeded)",
            "impl": "reference",
            "config": {"workload": WORKLOAD, "step": "40 channels x 2^18 samples (bounded sample of a block)"},
            "cpu_baseline": {"value": v, "unit": "channel-MS/s", "cores": threads, "kind": "port",
                             "sample": f"40 channels x {args.steps} x 2^18 samples"},
            "e2e": {"value": v, "unit": "channel-MS/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    barrier(world)


def pipelined(runner, inputs):
    """Submit every block with two in flight; each block's outputs are in host
    memory (or the device arena) after its wait."""
    prev = None
    for x in inputs:
        t = runner.submit(x)
        if prev is not None:
            runner.wait(prev)
        prev = t
    if prev is not None:
        runner.wait(prev)


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch

    import gpudemod as G
    world, rank, local = dist_setup(args.gpus)
    dev = torch.device("cuda", local)
    # one continuous stream: the value pass, then the e2e pass, without a jump
    # back in the input (which would make every pilot loop re-acquire)
    n_scene = min(max(N_BLOCKS, 2 * (args.warmup + args.steps)), 160)
    blocks, stations = make_scene(dev, rank, n_blocks=n_scene)
    torch.cuda.synchronize()

    runner = G.ChannelRunner(FS, BLOCK, max_channels=64, max_taps=1024)
    admit_all(runner, stations)
    stream = torch.cuda.ExternalStream(runner.stream_handle(), device=dev)
    work = algorithmic_work()

    # ---- value: inputs resident in HBM, outputs kept on the device ----------
    runner.set_host_outputs(False)
    runner.set_profiling(True)
    clk = ClockSampler(local).__enter__()  # sampling starts before warmup (first sample ~0.2 s)
    pipelined(runner, [blocks[s % n_scene] for s in range(args.warmup)])
    runner.reset_stats()
    l0 = G.kernel_launch_count()
    stage_acc = {}
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)  # the runner's join stream: events there follow every submitted block
    prev = None
    for s in range(args.steps):
        t = runner.submit(blocks[(args.warmup + s) % n_scene])  # two blocks in flight
        if prev is not None:
            runner.wait(prev)
            for name, ms in runner.stage_times():
                stage_acc.setdefault(name, []).append(ms)
        prev = t
    runner.wait(prev)
    for name, ms in runner.stage_times():
        stage_acc.setdefault(name, []).append(ms)
    e1.record(stream)
    torch.cuda.synchronize()
    launches = G.kernel_launch_count() - l0
    pll_paths = [runner.result(sl, payload=False) for sl in range(N_CH)]
    pll_info = {"parallel_blocks": sum(1 for r in pll_paths if r["pll_path"] == 1), "channels": N_CH,
                "newton_iters": sorted({r["pll_iters"] for r in pll_paths})}
    t_ms = max_over_ranks(world, e0.elapsed_time(e1))
    barrier(world)
    value = world * N_CH * BLOCK * args.steps / (t_ms * 1e-3) / 1e6
    st_value = runner.stats()

    # ---- e2e: public C ABI from pinned host memory ---------------------------
    runner.set_profiling(False)
    runner.set_host_outputs(True)
    # the next warmup + steps blocks of the stream, in pinned host memory
    first = args.warmup + args.steps
    pinned = [blocks[(first + b) % n_scene].cpu().pin_memory() for b in range(args.warmup + args.steps)]
    pipelined(runner, pinned[:args.warmup])
    runner.reset_stats()
    barrier(world)
    torch.cuda.synchronize()
    e0.record(stream)
    pipelined(runner, pinned[args.warmup:])
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(world, e0.elapsed_time(e1)) * 1e-3
    clk.__exit__(None, None, None)
    clocks = clk.summary()
    st = runner.stats()
    e2e = world * N_CH * BLOCK * args.steps / e2e_s / 1e6
    h2d, d2h = st["last_h2d_bytes"], st["last_d2h_bytes"]

    result = None
    if rank == 0:
        # ---- plain per-signal runner on the same GPU ---------------------
        plain_v = None
        if not args.profile_only and args.plain_steps > 0:
            pr = G.ChannelRunner(FS, BLOCK, max_channels=64, max_taps=1024)
            admit_all(pr, stations)
            pr.set_schedule(G.SCHED_PLAIN)
            pr.process_block(blocks[0])
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for s in range(args.plain_steps):
                pr.process_block(blocks[1 + s])
            plain_s = time.perf_counter() - t0
            plain_v = N_CH * BLOCK * args.plain_steps / plain_s / 1e6
            pr.close()

        # ---- roofline of the dominant kernel ----------------------------
        hbm_peak, peak_kind = measured_peaks()
        fp32 = fp32_peak_tflops() if not args.profile_only else None
        # per-launch device time of each kernel; the intervals that cover a
        # wait on the other block in flight and the copies are not kernels
        kern = {k: statistics.mean(v) for k, v in stage_acc.items()
                if k not in ("h2d", "d2h") and not k.startswith("wait")}
        waits = {k: round(statistics.mean(v), 4) for k, v in stage_acc.items() if k.startswith("wait")}
        dom = max(kern, key=kern.get)
        dom_key = "extract" if dom.startswith("extract") else ("pll" if dom.startswith("pll") else dom)
        w = work.get(dom_key, {"flop": 0, "bytes": 0})
        dom_ms = kern[dom]
        ach_tf = w["flop"] / (dom_ms * 1e-3) / 1e12
        ach_gbs = w["bytes"] / (dom_ms * 1e-3) / 1e9
        fp32_bound = fp32 is not None and (w["flop"] / (fp32 * 1e12)) >= (w["bytes"] / (hbm_peak * 1e9))
        if fp32_bound:
            roof = {"bound": "fp32", "achieved": ach_tf, "peak": fp32, "unit": "TFLOP/s", "frac": ach_tf / fp32,
                    "peak_source": "cuBLAS SGEMM (TF32 off), measured in this run"}
        else:
            roof = {"bound": "hbm", "achieved": ach_gbs, "peak": hbm_peak, "unit": "GB/s",
                    "frac": ach_gbs / hbm_peak, "peak_source": f"{peak_kind} HBM copy"}
        roof.update({"kernel": dom, "ms_per_launch": dom_ms, "traffic": None,
                     "algorithmic_flop": w["flop"], "algorithmic_bytes": w["bytes"],
                     "hbm_frac": ach_gbs / hbm_peak})
        block_ms_sum = sum(kern.values())
        stages = {k: round(v, 4) for k, v in sorted(kern.items(), key=lambda kv: -kv[1])}

        # ---- CPU baseline (oracle port), bounded sample ---------------------
        cpu = None
        if not args.no_cpu and not args.profile_only:
            nb = args.cpu_blocks
            bnp = [blocks[b].cpu().numpy() for b in range(nb)]
            threads = host_threads()
            v, dt = cpu_run(bnp, stations, nb, threads)
            cpu = {"value": v, "unit": "channel-MS/s", "cores": threads, "kind": "port",
                   "sample": f"{N_CH} channels x {nb} blocks of 2^20 through the oracle chain ({dt:.1f} s wall)"}

        total_flop = work["per_block_flop"]
        result = {
            "metric": METRIC, "value": value, "unit": "channel-MS/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 NCO/PLL state)",
            "data": "synthetic (seeded scene, stands in for live captures)",
            "config": {"workload": WORKLOAD, "channels": N_CH, "block": BLOCK, "taps": TAPS, "decim": FS // OUT_RATE,
                       "inputs": f"{n_scene} consecutive 8 MiB blocks of one continuous stream resident in HBM "
                                 f"({n_scene * 8} MiB > L2); the e2e pass continues the stream from pinned host memory",
                       "parallelism": f"channel shards, {world} GPU(s), no data-path collective"},
            "e2e": {"value": e2e, "unit": "channel-MS/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "p50_block_ms": st["p50_block_ms"], "p99_block_ms": st["p99_block_ms"]},
            "plain_runner": {"value": plain_v, "unit": "channel-MS/s",
                             "speedup_batched_vs_plain": (value / plain_v) if plain_v else None},
            "latency_ms": {"p50": st_value["p50_block_ms"], "p99": st_value["p99_block_ms"],
                           "block_period_ms": BLOCK / FS * 1e3},
            "roofline": roof,
            "stage_ms": stages,
            "wait_ms": waits,
            "block_gflop": total_flop / 1e9,
            "block_tflops": total_flop / (block_ms_sum * 1e-3) / 1e12,
            "cpu_baseline": cpu,
            "gpu_launches": launches,
            "pll": pll_info,
            "clocks": clocks,
        }
    runner.close()
    barrier(world)
    if rank == 0:
        print(json.dumps(result))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
