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
             runner's launches over the timed region (three blocks in flight,
             so an interval includes the other blocks' kernels sharing SMs);
             extraction_rooflines: every extraction kernel the same way;
             rooflines_one_block_in_flight: the same from a short pass with one
             block in flight after the timed passes
  e2e.h2d_gbs  the pinned copy of one input block timed alone; h2d_bound the
             e2e value that copy rate alone would allow
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
E2E_MIN_BLOCKS = 96  # e2e pass: blocks timed through the public API from pinned host memory
TAPS = 256
OUT_RATE = 312_500
BW = 250_000.0
N_BLOCKS = 64
METRIC = "aggregate channel-MS/s on 1 B200 (serving vs plain runner); p99 block latency"
WORKLOAD = ("FM band batch: 10 MS/s cf32, 2^20-sample blocks, 40 WFM stations on a 200 kHz grid "
            "(10-40 dB SNR), 256-tap FIR, decimate by 32 to 312.5 kS/s, FM discriminator, stereo "
            "decode with 19 kHz pilot PLL, RDS baseband; audio returned as the streaming path delivers "
            "it: 48 kHz stereo s16le (polyphase resample, 50 us de-emphasis, x0.35)")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--plain-steps", type=int, default=3)
    ap.add_argument("--depth", type=int, default=3, help="blocks in flight (the runner holds three frames)")
    ap.add_argument("--cpu-blocks", type=int, default=8, help="cpu_baseline sample: blocks of 2^20 per channel")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--iso-blocks", type=int, default=8, help="blocks timed kernel by kernel with one in flight")
    ap.add_argument("--backend", default="nccl", choices=["nccl", "gloo"])
    ap.add_argument("--plan-only", action="store_true",
                    help="form the process world and print the channel shards (no GPU work)")
    ap.add_argument("--no-serving", action="store_true", help="fm_band: leave out the serving phases")
    ap.add_argument("--no-autotune", action="store_true", help="mixed: keep the runner's static form rule")
    ap.add_argument("--profile-only", action="store_true", help="short run for ncu (no baselines)")
    ap.add_argument("--workload", default="fm_band", choices=["fm_band", "mixed", "serving", "headroom"],
                    help="fm_band: the FM band batch (headline); mixed: the mixed-mode uneven batch; "
                         "serving: the serving request stream; headroom: 2048 channels at 61.44 MS/s with churn")
    ap.add_argument("--headroom-channels", type=int, default=2048)
    ap.add_argument("--serve-seconds", type=float, default=8.0, help="serving: seconds of stream per phase")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# standalone helpers: the scene generator (gpudemod/synth.py) and the process
# plumbing (gpudemod/dist.py) import nothing from the package, so they are
# loaded by file path.  Importing the gpudemod package itself loads the CUDA
# library, which the reference arm must not map.
# ---------------------------------------------------------------------------
def standalone(mod: str):
    import importlib.util
    name = f"_gpudemod_{mod}_standalone"
    if name not in sys.modules:
        spec = importlib.util.spec_from_file_location(name, os.path.join(ROOT, "argus-sdr_b200", "gpudemod",
                                                                         f"{mod}.py"))
        m = importlib.util.module_from_spec(spec)
        sys.modules[name] = m
        spec.loader.exec_module(m)
    return sys.modules[name]


# ---------------------------------------------------------------------------
# distributed plumbing: one process per GPU (torchrun's environment, or the
# ranks this script spawns itself for --gpus N), channels sharded by the cost
# model, no data-path collective: a barrier and a max-reduction of timings only
# ---------------------------------------------------------------------------
def dist_setup(args):
    D = standalone("dist")
    world, rank, local = D.init(args.backend)
    if world != args.gpus:
        raise SystemExit(f"--gpus {args.gpus} but the process world has {world} rank(s)")
    return world, rank, local


def barrier(world):
    standalone("dist").barrier(world)


def max_over_ranks(world, v: float, device="cuda") -> float:
    return standalone("dist").max_over_ranks(world, v, device=device)


def spawn_ranks(args) -> int:
    """--gpus N outside torchrun: start N copies of this command, one per
    GPU, as torchrun would (RANK / LOCAL_RANK / WORLD_SIZE / MASTER_* on
    127.0.0.1); rank 0 prints the line.  Returns the first nonzero exit code."""
    import socket
    import subprocess
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    procs = []
    for r in range(args.gpus):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(args.gpus),
                   LOCAL_WORLD_SIZE=str(args.gpus), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, os.path.abspath(__file__)] + sys.argv[1:], env=env))
    rcs = [p.wait() for p in procs]
    return next((rc for rc in rcs if rc), 0)


def channel_shard(costs, world, rank):
    """This rank's channel indices: longest-processing-time-first over the
    per-channel cost model (every rank computes the same partition)."""
    return standalone("dist").partition_channels(costs, world)[rank]


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
def make_scene(device, n_blocks=N_BLOCKS):
    """The FM band scene: one continuous seeded stream, the same on every rank
    (each rank extracts its own shard of the channels from the same blocks)."""
    import torch

    synth = standalone("synth")
    scene, stations = synth.fm_band_scene(device=device, block=BLOCK, n_stations=N_CH,
                                          seconds=n_blocks * BLOCK / FS + 1, seed=synth.CONFIG_SEEDS[1])
    blocks = torch.empty((n_blocks, BLOCK), dtype=torch.complex64, device=device)
    for b in range(n_blocks):
        blocks[b] = scene.next_block()
    return blocks, stations


def fm_band_shard(stations, world, rank):
    """Weak scaling over channel shards: the job's channel set is the 40
    stations once per GPU (signal id copy * 40 + station), partitioned over
    the ranks by the per-channel cost model, so every GPU extracts 40
    channels from the same wideband block.  Returns [(signal_id, station)]."""
    D = standalone("dist")
    chans = [(c * N_CH + i, st) for c in range(world) for i, st in enumerate(stations)]
    cost = D.channel_cost(BLOCK, FS // OUT_RATE, TAPS, 3)
    return [chans[i] for i in channel_shard([cost] * len(chans), world, rank)]


def admit_all(runner, shard):
    import gpudemod as G
    return [runner.admit(sid, st.offset_hz, BW, OUT_RATE, TAPS, G.MODE_WFM_STEREO, G.CH_RDS | G.CH_AUDIO48K)
            for sid, st in shard]


def fm_band_channels():
    return [dict(kind="WFM", T=TAPS, D=FS // OUT_RATE, out_rate=OUT_RATE) for _ in range(N_CH)]


def extraction_form(T, D):
    """The runner's choice of extraction kernel for a channel (host
    choose_extraction): arms of <= 4 taps take the modulated form, else the
    dense kernel when a 256-output tile's D phases fit in 200 KB of shared
    memory, else phase groups."""
    P, L = min(D, T), -(-T // D)
    if L <= 4:
        return "extract_mod"
    M = 256 + L - 1
    Mp = (M + (M >> 3) + 1) | 1
    z = max((P * Mp * 8 + 15) & ~15, 8 * 288 * 16)
    smem = z + ((P * L + 3) & ~3) * 4 + ((P * (256 + L - 1) + 255) // 256) * 8 + 16
    return "extract_dense" if L <= 16 and smem <= 200 * 1024 else "extract_group"


def gemm_grouped(chans, n_in=BLOCK):
    """Indices of the channels the runner extracts as tensor-core channel
    groups (host plan_gemm_groups): dense-form channels whose decimation is a
    multiple of 4, not float64-summed (FM modes at >= 4x their bandwidth),
    with more than 256 outputs, in (taps, decimation) classes of at least 4
    channels (all channels of a workload share the phase count here: they are
    admitted together and every block length is a multiple of the
    decimation).  Also returns the executed tensor flop per block: three TF32
    passes of a 128 x N x 2*L*D real GEMM per 128-output tile."""
    classes = {}
    for i, c in enumerate(chans):
        T, D = c["T"], c["D"]
        fm = c["kind"] in ("NFM", "WFM")
        precise = fm and c.get("bw") is not None and c["out_rate"] >= 4 * max(c["bw"], 400.0)
        if (c.get("form") or extraction_form(T, D)) != "extract_dense" or D % 4 or precise or n_in // D <= 256:
            continue
        classes.setdefault((T, D), []).append(i)
    grouped, tensor_flop = set(), 0
    for (T, D), idx in classes.items():
        if len(idx) < 4:
            continue
        L = -(-T // D)
        rp = ((128 + L - 1 + 7) // 8) * 8 + 1
        smem = lambda n, ns: 128 + 128 * 24 + 2 * (D // 2) * rp * 16 + ns * 2 * (D // 2) * n * 16
        cmax = max([c for c in range(8, 129, 8) if smem(2 * c, 2) <= 220 * 1024] or [0])
        if cmax < 4:
            continue
        nchunk = -(-len(idx) // cmax)
        per = -(-len(idx) // nchunk)
        for c0 in range(0, len(idx), per):
            members = idx[c0:c0 + per]
            if len(members) < 4:
                break
            grouped.update(members)
            ncol = -(-2 * len(members) // 16) * 16
            tiles = -(-(n_in // D - 256) // 128)
            tensor_flop += 3 * 2 * 128 * ncol * 2 * L * D * tiles
    return grouped, tensor_flop


def bank_grouped(chans, n_in=BLOCK, grouped=()):
    """Channels the runner extracts as short-arm channel banks (host
    plan_bank_groups): warp-per-output or modulated-form channels with at
    most four taps per arm, not float64-summed, not in a tensor-core group,
    in (taps, decimation) classes of at least 4 (the workloads admit every
    channel together, so they share the phase count).  Returns {index: first
    banked output}."""
    classes = {}
    for i, c in enumerate(chans):
        T, D = c["T"], c["D"]
        fm = c["kind"] in ("NFM", "WFM")
        precise = fm and c.get("bw") is not None and c["out_rate"] >= 4 * max(c["bw"], 400.0)
        form = c.get("form") or extraction_form(T, D)
        if i in grouped or form not in ("extract_wide", "extract_mod") or precise or -(-T // D) > 4:
            continue
        classes.setdefault((T, D), []).append(i)
    out = {}
    for (T, D), idx in classes.items():
        if len(idx) < 4:
            continue
        s0 = D - 1  # phase count 0 at the first block; every block here is a multiple of D or close to it
        jb = -(-(T - 1 - s0) // D) if T - 1 > s0 else 0
        if n_in // D > jb:
            out.update({i: jb for i in idx})
    return out


def algorithmic_work(chans, n_in=BLOCK):
    """Algorithmic work per block, summed over channels: extraction
    4*T*n_out + min(6*n_in, 4*T*n_out) flop (complex x real taps, plus the
    cheaper of a rotation per input sample or modulated taps); discriminator
    6, AM 5, SSB 3, CW 1 flop per output; WFM composite: the reference's six
    101-tap FIRs at 2 flop per tap + PLL ~36 per sample; RDS 4*101 per RDS
    output + 2 per composite sample; 48 kHz back end 2*33 per output frame and
    audio channel (+4 de-emphasis and gain for WFM).  Transcendentals count 0.
    Per-stage bytes are each stage's own reads and writes;
    block_min_bytes = the wideband block once + outputs + taps + history."""
    w = {k: {"flop": 0, "bytes": 0} for k in ("extract", "demod", "wfm_fir", "wfm_out", "pll", "rds", "audio48")}
    w["extract"]["bytes"] = 8 * n_in
    forms = {}  # the same extraction work split by the kernel that does it
    per_out = {"WFM": 6, "NFM": 6, "AM": 5, "USB": 3, "LSB": 3, "CW": 1}
    grouped, tensor_flop = gemm_grouped(chans, n_in)
    banked = bank_grouped(chans, n_in, grouped)
    bmin = 8 * n_in  # the wideband block, read once for all channels
    for i, c in enumerate(chans):
        T, D = c["T"], c["D"]
        n_out = n_in // D
        f = 4 * T * n_out + min(6 * n_in, 4 * T * n_out)
        b = 8 * n_out + 4 * T + 16 * (T - 1)
        w["extract"]["flop"] += f
        w["extract"]["bytes"] += b
        if i in grouped:
            # outputs 0..255 (the carried history) on the dense kernel, the rest in the group kernel
            f0 = f * 256 / n_out
            fw = forms.setdefault("extract_dense", {"flop": 0, "bytes": 8 * n_in})
            fw["flop"] += f0
            fw["bytes"] += 8 * 256
            fw = forms.setdefault("extract_gemm", {"flop": 0, "bytes": 8 * n_in, "tensor_flop": tensor_flop})
            fw["flop"] += f - f0
            fw["bytes"] += b - 8 * 256
        elif i in banked:
            # outputs before the bank's first tile (the carried history) on the warp-per-output kernel
            f0 = f * banked[i] / n_out
            fw = forms.setdefault("extract_wide", {"flop": 0, "bytes": 8 * n_in})
            fw["flop"] += f0
            fw["bytes"] += 8 * banked[i]
            fw = forms.setdefault("extract_bank", {"flop": 0, "bytes": 8 * n_in})
            fw["flop"] += f - f0
            fw["bytes"] += b - 8 * banked[i]
        else:
            fw = forms.setdefault(c.get("form") or extraction_form(T, D), {"flop": 0, "bytes": 8 * n_in})
            fw["flop"] += f
            fw["bytes"] += b
        w["demod"]["flop"] += per_out[c["kind"]] * n_out
        w["demod"]["bytes"] += 12 * n_out
        # 48 kHz back end: 33-tap arm per output frame and audio channel,
        # de-emphasis 3 and gain 1 per sample (WFM); 2 bytes per PCM sample
        ach = 2 if c["kind"] == "WFM" else 1
        if c.get("pcm", True):
            n48 = n_out * 48000 // c["out_rate"]
            w["audio48"]["flop"] += ach * n48 * (2 * 33 + (4 if c["kind"] == "WFM" else 0))
            w["audio48"]["bytes"] += ach * (n_out * 4 + n48 * 2)
        if c["kind"] == "WFM":
            dr = c["out_rate"] // 19000
            n_rds = n_out // dr
            # the reference's stereo decoder runs six 101-tap FIRs per composite
            # sample (L+R 15k, 53k, 23k, 21k, 17k here; L-R 15k in wfm_out);
            # the kernel differences the band-pass pairs' taps and runs three
            w["wfm_fir"]["flop"] += 5 * 2 * 101 * n_out
            w["wfm_fir"]["bytes"] += 16 * n_out
            w["wfm_out"]["flop"] += 2 * 101 * n_out
            w["wfm_out"]["bytes"] += 16 * n_out
            w["pll"]["flop"] += 36 * n_out
            w["pll"]["bytes"] += 12 * n_out
            w["rds"]["flop"] += 404 * n_rds + 2 * n_out
            w["rds"]["bytes"] += 4 * n_out + 8 * n_rds
        # minimum bytes: outputs (8 B per stereo frame or IQ sample, 4 B per
        # mono audio sample, 8 B per RDS sample) + taps read + history read/write
        if c["kind"] == "WFM":
            ob = 8 * n_out + 8 * (n_out // (c["out_rate"] // 19000))
        else:
            ob = 4 * n_out
        bmin += ob + 4 * T + 16 * (T - 1)
    w["per_block_flop"] = sum(v["flop"] for v in w.values())
    w["block_min_bytes"] = bmin
    w.update(forms)
    return w


def stage_key(name):
    """Work group of a runner stage name (extraction by kernel form)."""
    if name.startswith("extract_dense"):
        return "extract_dense"
    if name == "extract_group":
        return "extract_group"
    if name in ("extract_bank", "bank_pack"):
        return "extract_bank"
    if name.startswith("extract"):
        return name
    if name.startswith("pll"):
        return "pll"
    if name in ("demod", "am"):
        return "demod"
    if name == "audio48k":
        return "audio48"
    return name


# DRAM bytes (read + write) per launch, by runner stage, from ncu captures of
# the kernel on the same workload (cold cache, serialised); None where no
# capture exists.
NCU_TRAFFIC = {("fm_band", "extract_gemm"): 8.73e6,
               ("fm_band", "pll"): 10.58e6,
               }
# Headroom stress, captured at 512 channels (the 2048-channel launch was not
# captured): the phase-group kernels read the L2-resident block once and write
# nothing to DRAM during the launch, so their traffic does not grow with the
# channel count and is reported as measured, not scaled.
NCU_TRAFFIC_HEADROOM_512 = {"extract_mod": 10.23e6, "extract_group": 9.70e6}


def kernel_roofline(name, ms, work, fp32, hbm_peak, peak_kind, wl, tf32=None):
    """Roofline entry of one runner stage from its per-launch device time:
    the algorithmic work of its channels (the definitions of
    algorithmic_work) against the FP32 FMA peak or the HBM peak, whichever
    takes longer for that work; frac = achieved / that peak.  The
    tensor-core group kernel also reports its executed TF32 work against the
    measured TF32 GEMM rate, as context."""
    key = stage_key(name)
    w = work.get(key, {"flop": 0, "bytes": 0})
    sec = ms * 1e-3
    t_flop = w["flop"] / (fp32 * 1e12)
    t_byte = w["bytes"] / (hbm_peak * 1e9)
    if t_flop >= t_byte:
        ach = w["flop"] / sec / 1e12
        roof = {"bound": "fp32", "achieved": ach, "peak": fp32, "unit": "TFLOP/s", "frac": ach / fp32,
                "peak_source": "FP32 FMA microbenchmark, measured in this run"}
    else:
        ach = w["bytes"] / sec / 1e9
        roof = {"bound": "hbm", "achieved": ach, "peak": hbm_peak, "unit": "GB/s", "frac": ach / hbm_peak,
                "peak_source": f"{peak_kind} HBM copy (MEASURED_PEAKS.json)"}
    traffic = NCU_TRAFFIC.get((wl, key))
    roof.update({"kernel": name, "ms_per_launch": ms, "traffic": traffic,
                 "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, one launch" if traffic else None,
                 "algorithmic_flop": w["flop"], "algorithmic_bytes": w["bytes"],
                 "roofline_ms": max(t_flop, t_byte) * 1e3})
    if "tensor_flop" in w and tf32:
        roof["tensor_context"] = {"executed_tf32_flop": w["tensor_flop"],
                                  "tflops": w["tensor_flop"] / sec / 1e12, "tf32_gemm_tflops": tf32}
    return roof


def h2d_rate(block):
    """Host-to-device copy rate (GB/s) of one pinned input block, timed
    alone on a stream of its own (not the runner's: torch's pinned-memory
    allocator records every stream a pinned block was copied on, and records
    an event there when the block is freed, which may be after the runner
    has gone): the bound of any e2e number whose every block crosses the
    host link."""
    import torch
    dst = torch.empty_like(block, device="cuda")
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        for _ in range(2):
            dst.copy_(block, non_blocking=True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(10):
            dst.copy_(block, non_blocking=True)
        e1.record(stream)
    torch.cuda.synchronize()
    return 10 * block.numel() * block.element_size() / (e0.elapsed_time(e1) * 1e-3) / 1e9


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def fp32_fma_peak():
    """FP32 FMA rate of this GPU from the committed microbenchmark
    (csrc/fma_peak.cu: eight independent fmaf chains per thread, 8 CTAs of 256
    threads per SM): (TFLOP/s, kernel ms)."""
    import ctypes as C
    lib = C.CDLL(os.path.join(ROOT, "argus-sdr_b200", "libgpudemod_peak.so"))
    tf, ms = C.c_double(), C.c_double()
    rc = lib.gpud_peak_fp32_fma(16384, 8, 5, C.byref(tf), C.byref(ms))
    if rc != 0:
        raise RuntimeError(f"gpud_peak_fp32_fma failed: {rc}")
    return tf.value, ms.value


def tf32_gemm_tflops():
    """cuBLAS TF32 GEMM 8192^3 rate (context for the tensor-core group kernel)."""
    import torch
    torch.backends.cuda.matmul.allow_tf32 = True
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
    torch.backends.cuda.matmul.allow_tf32 = False
    return 2 * 8192 ** 3 / (best * 1e-3) / 1e12


# ---------------------------------------------------------------------------
# CPU path (oracle restatement of the reference's Go CPU code)
# ---------------------------------------------------------------------------
class CpuChannel:
    """The reference's CPU path for one channel: the oracle chain, then the
    48 kHz back end (resample, de-emphasis, gain, s16le) on its audio."""

    def __init__(self, O, fs, off, bw, rate, taps, mode, kind, rds):
        self.ch = O.OracleChannel(fs, off, bw, rate, taps, mode, rds=rds)
        stereo = mode == O.MODE_WFM_STEREO
        self.back = O.Audio48(rate, 2 if stereo else 1, wfm=kind == "WFM", deemph_us=50.0)

    def process(self, x):
        out = self.ch.process(x)
        self.back.process(out["audio"])


def cpu_channels(stations):
    from oracle import oracle as O
    return [CpuChannel(O, FS, st.offset_hz, BW, OUT_RATE, TAPS, O.MODE_WFM_STEREO, "WFM", True) for st in stations]


def cpu_run(blocks_np, chans, threads):
    """Every channel through every block in order (state carried), channels
    spread over `threads` host threads.  Returns (channel-MS/s, seconds)."""
    def work(c):
        for x in blocks_np:
            c.process(x)

    t0 = time.perf_counter()
    if threads == 1:
        for c in chans:
            work(c)
    else:
        with cf.ThreadPoolExecutor(max_workers=threads) as ex:
            list(ex.map(work, chans))
    dt = time.perf_counter() - t0
    return len(chans) * len(blocks_np) * BLOCK / dt / 1e6, dt


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_model():
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def fm_band_config(world):
    """The FM band workload's config, identical in both arms."""
    return {"workload": WORKLOAD, "channels": N_CH * world, "channels_per_gpu": N_CH, "block": BLOCK,
            "taps": TAPS, "decim": FS // OUT_RATE, "step": f"one 2^20-sample block through all {N_CH * world} "
                                                           f"channels",
            "parallelism": f"channel shards over {world} GPU(s) by the cost model, no data-path collective"}


# ---------------------------------------------------------------------------
def run_reference(args):
    """The reference's CPU path for this workload: the oracle port of the Go
    CPU chain (extraction, discriminator, stereo decoder with pilot PLL, RDS
    baseband) plus the 48 kHz audio back end, one channel per task on all host
    threads.  A step is the same step as the GPU arm's: one 2^20-sample block
    of the same continuous stream through all 40 channels.  Under torchrun
    only rank 0 runs; nothing here loads the CUDA library."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    import torch
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    nb = args.warmup + args.steps
    blocks, stations = make_scene(dev, n_blocks=nb)
    blocks_np = [b.cpu().numpy() for b in blocks]
    del blocks
    threads = host_threads()
    chans = cpu_channels(stations)
    for b in range(args.warmup):
        cpu_run([blocks_np[b]], chans, threads)
    dt = 0.0
    for b in range(args.steps):
        dt += cpu_run([blocks_np[args.warmup + b]], chans, threads)[1]
    v = N_CH * BLOCK * args.steps / dt / 1e6
    line = {"metric": METRIC, "value": v, "unit": "channel-MS/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 NCO/PLL state)",
            "data": "synthetic (seeded scene, stands in for live captures)", "impl": "reference",
            "config": fm_band_config(1),
            "cpu_baseline": {"value": v, "unit": "channel-MS/s", "cores": threads, "kind": "port",
                             "cpu_model": cpu_model(),
                             "sample": f"{N_CH} channels x {args.steps} consecutive 2^20-sample blocks (the full "
                                       f"step, not a sample) through the C restatement of the reference's Go CPU "
                                       f"path + 48 kHz back end"},
            "e2e": {"value": v, "unit": "channel-MS/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def pipelined(runner, inputs, depth=3):
    """Submit every block with up to `depth` in flight; each block's outputs
    are in host memory (or the device arena) after its wait."""
    tickets = []
    for x in inputs:
        tickets.append(runner.submit(x))
        if len(tickets) >= depth:
            runner.wait(tickets[-depth])
    if tickets:
        runner.wait(tickets[-1])


def measure_batch(args, world, rank, local, runner, blocks, n_scene, chans, wl, make_plain, cpu_baseline):
    """value (inputs in HBM, `depth` blocks in flight), e2e (pinned host
    memory through the public API), per-kernel times with one block in
    flight, the plain per-signal runner, the roofline of the dominant kernel
    and of the whole block, and the CPU baseline, for one batch workload."""
    import torch

    import gpudemod as G
    dev = torch.device("cuda", local)
    n_ch = len(chans)
    stream = torch.cuda.ExternalStream(runner.stream_handle(), device=dev)
    work = algorithmic_work(chans)

    # the e2e pass's blocks (the stream after the value pass's) in pinned host
    # memory, prepared up front so that the GPU does not idle between the passes
    first = args.warmup + args.steps
    e2e_steps = max(args.steps, E2E_MIN_BLOCKS)
    pool = [blocks[(first + b) % n_scene].cpu().pin_memory() for b in range(min(n_scene, args.warmup + e2e_steps))]
    pinned = [pool[b % len(pool)] for b in range(args.warmup + e2e_steps)]

    # ---- value: inputs resident in HBM, outputs kept on the device ----------
    runner.set_host_outputs(False)
    clk = ClockSampler(local).__enter__()  # sampling starts before warmup (first sample ~0.2 s)
    pipelined(runner, [blocks[s % n_scene] for s in range(args.warmup)], args.depth)
    runner.reset_stats()
    l0 = G.kernel_launch_count()
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)  # the runner's join stream: events there follow every submitted block
    pipelined(runner, [blocks[(args.warmup + s) % n_scene] for s in range(args.steps)], args.depth)
    e1.record(stream)
    torch.cuda.synchronize()
    launches = G.kernel_launch_count() - l0
    wfm_slots = [i for i, c in enumerate(chans) if c["kind"] == "WFM"]
    pll_info = None
    if wfm_slots:
        res = [runner.result(sl, payload=False) for sl in wfm_slots]
        pll_info = {"parallel_blocks": sum(1 for r in res if r["pll_path"] == 1), "channels": len(wfm_slots),
                    "newton_iters": sorted({r["pll_iters"] for r in res})}
    t_ms = max_over_ranks(world, e0.elapsed_time(e1))
    barrier(world)
    value = world * n_ch * BLOCK * args.steps / (t_ms * 1e-3) / 1e6
    st_value = runner.stats()

    # ---- e2e: public C ABI from pinned host memory ---------------------------
    runner.set_host_outputs(True)
    pipelined(runner, pinned[:args.warmup], args.depth)
    runner.reset_stats()
    barrier(world)
    torch.cuda.synchronize()
    e0.record(stream)
    pipelined(runner, pinned[args.warmup:], args.depth)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(world, e0.elapsed_time(e1)) * 1e-3
    clk.__exit__(None, None, None)
    clocks = clk.summary()
    st = runner.stats()
    e2e = world * n_ch * BLOCK * e2e_steps / e2e_s / 1e6
    h2d, d2h = st["last_h2d_bytes"], st["last_d2h_bytes"]
    # the host link during the pass: every block's copy into the input ring
    # is timed on the copy stream
    ring_ms = st["ring_copy_ms"] / max(1, st["ring_copies"])
    link = {"ring_copies": st["ring_copies"], "copy_ms_per_block": ring_ms,
            "gbs_during_pass": (BLOCK * 8) / (ring_ms * 1e-3) / 1e9 if ring_ms > 0 else None,
            "busy_frac": st["ring_copy_ms"] / (e2e_s * 1e3),
            "bound": world * n_ch * BLOCK / (ring_ms * 1e-3) / 1e6 if ring_ms > 0 else None}
    h2d_gbs = h2d_rate(pinned[0])
    del pinned, pool
    if rank != 0:
        return None

    # ---- per-kernel device time with one block in flight: each interval
    # between the runner's stage events covers that kernel alone (with three
    # blocks in flight an interval would include the other blocks' kernels)
    iso_acc = {}
    runner.set_host_outputs(False)
    runner.set_profiling(True)
    nxt = first + args.warmup + args.steps  # the stream continues after the e2e pass
    for b in range(args.iso_blocks + 1):
        runner.process_block(blocks[(nxt + b) % n_scene])
        if b:
            for name, ms in runner.stage_times():
                iso_acc.setdefault(name, []).append(ms)
    runner.set_profiling(False)

    # ---- plain per-signal runner on the same GPU -------------------------
    plain_v = None
    if not args.profile_only and args.plain_steps > 0:
        pr = make_plain()
        pr.set_schedule(G.SCHED_PLAIN)
        pr.process_block(blocks[0])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for s in range(args.plain_steps):
            pr.process_block(blocks[1 + s])
        plain_s = time.perf_counter() - t0
        plain_v = n_ch * BLOCK * args.plain_steps / plain_s / 1e6
        pr.close()

    # ---- rooflines: the dominant kernel and the whole block -----------------
    hbm_peak, peak_kind = measured_peaks()
    fp32, fma_ms = fp32_fma_peak()
    tf32 = tf32_gemm_tflops() if (not args.profile_only and "extract_gemm" in work) else None
    kern = {k: statistics.median(v) for k, v in iso_acc.items() if k not in ("h2d", "d2h") and not k.startswith("wait")}
    dom = max(kern, key=kern.get)
    roof = kernel_roofline(dom, kern[dom], work, fp32, hbm_peak, peak_kind, wl, tf32)
    others = {k: {kk: (round(vv, 5) if isinstance(vv, float) else vv)
                  for kk, vv in kernel_roofline(k, v, work, fp32, hbm_peak, peak_kind, wl, tf32).items()
                  if kk in ("bound", "achieved", "frac", "ms_per_launch", "traffic")}
              for k, v in sorted(kern.items(), key=lambda kv: -kv[1]) if k != dom and stage_key(k) in work}
    total_flop = work["per_block_flop"]
    b_min = work["block_min_bytes"]
    t_roof = max(total_flop / (fp32 * 1e12), b_min / (hbm_peak * 1e9)) * 1e3
    block = {"gflop": total_flop / 1e9, "min_bytes": b_min, "roofline_ms": t_roof,
             "bound": "fp32" if total_flop / (fp32 * 1e12) >= b_min / (hbm_peak * 1e9) else "hbm",
             "measured_ms_per_block": t_ms / args.steps, "frac": t_roof / (t_ms / args.steps),
             "kernel_ms_one_block_in_flight": sum(kern.values())}

    # ---- CPU baseline (oracle port), bounded sample -------------------------
    cpu = None
    if not args.no_cpu and not args.profile_only:
        cpu = cpu_baseline(blocks)

    return {
        "value": value, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 NCO/PLL state)",
        "data": "synthetic (seeded scene, stands in for live captures)",
        "e2e": {"value": e2e, "unit": "channel-MS/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "h2d_gbs": h2d_gbs,
                "h2d_bound": world * n_ch * BLOCK / (h2d / (h2d_gbs * 1e9)) / 1e6,
                "host_link_during_pass": link,
                "p50_block_ms": st["p50_block_ms"], "p99_block_ms": st["p99_block_ms"],
                "blocks_timed": e2e_steps,
                "note": f"{e2e_steps} consecutive blocks (at least {E2E_MIN_BLOCKS}, so that the window is steady), "
                        f"{args.depth} in flight, each copied from pinned host memory into the runner's input ring "
                        f"and its outputs read back into pinned host memory; h2d_gbs is one block's copy timed "
                        f"alone, host_link_during_pass the copies as they ran inside the pass"},
        "plain_runner": {"value": plain_v, "unit": "channel-MS/s",
                         "speedup_batched_vs_plain": (value / plain_v) if plain_v else None},
        "latency_ms": {"p50": st_value["p50_block_ms"], "p99": st_value["p99_block_ms"],
                       "block_period_ms": BLOCK / FS * 1e3},
        "roofline": roof,
        "roofline_block": block,
        "kernels_one_block_in_flight": others,
        "fp32_fma_peak": {"tflops": fp32, "kernel_ms": fma_ms},
        "cpu_baseline": cpu,
        "gpu_launches": launches,
        "pll": pll_info,
        "clocks": clocks,
    }


def run_fm_band(args, world, rank, local):
    import torch

    import gpudemod as G
    dev = torch.device("cuda", local)
    # one continuous stream: the value pass, then the e2e pass, without a jump
    # back in the input (which would make every pilot loop re-acquire)
    n_scene = min(max(N_BLOCKS, 2 * (args.warmup + args.steps) + args.iso_blocks + 1), 160)
    blocks, stations = make_scene(dev, n_blocks=n_scene)
    torch.cuda.synchronize()
    shard = fm_band_shard(stations, world, rank)

    def make_runner():
        r = G.ChannelRunner(FS, BLOCK, max_channels=64, max_taps=1024)
        admit_all(r, shard)
        return r

    def cpu_baseline(blocks):
        nb = args.cpu_blocks
        bnp = [blocks[b].cpu().numpy() for b in range(nb)]
        threads = host_threads()
        v, dt = cpu_run(bnp, cpu_channels(stations), threads)
        n1 = 4  # single-thread sample: 4 stations
        v1, dt1 = cpu_run(bnp, cpu_channels(stations[:n1]), 1)
        return {"value": v, "unit": "channel-MS/s", "cores": threads, "kind": "port", "cpu_model": cpu_model(),
                "single_thread": v1,
                "sample": f"{N_CH} channels x {nb} consecutive blocks of 2^20 through the C restatement of the "
                          f"reference's Go CPU path + 48 kHz back end on {threads} threads ({dt:.1f} s wall); "
                          f"single thread: {n1} channels x {nb} blocks ({dt1:.1f} s)"}

    runner = make_runner()
    res = measure_batch(args, world, rank, local, runner, blocks, n_scene, fm_band_channels(), "fm_band",
                        make_runner, cpu_baseline)
    runner.close()
    del blocks
    torch.cuda.empty_cache()
    serving = None
    if not args.no_serving and not args.profile_only:
        out, plain, _, _ = serve_phases(args, world, rank, local, args.serve_seconds)
        serving = serving_summary(out, plain) if rank == 0 else None
    if res is None:
        return None
    line = {"metric": METRIC, "unit": "channel-MS/s"}
    line.update(res)
    line["serving"] = serving
    line["config"] = fm_band_config(world)
    line["inputs"] = (f"{n_scene} consecutive 8 MiB blocks of one continuous stream resident in HBM "
                      f"({n_scene * 8} MiB > L2); the e2e pass continues the stream from pinned host memory")
    return line


MIXED_WORKLOAD = ("Mixed-mode uneven batch: 10 MS/s cf32, 2^20-sample blocks, 120 channels at random "
                  "non-overlapping offsets, SNR 5-35 dB: 40 NFM (12.5 kHz, 512 taps, D 400), 30 AM (10 kHz, "
                  "384 taps, D 400), 30 SSB (3 kHz, 256 taps, D 800), 20 CW (500 Hz, 128 taps, D 2000)")


def run_mixed(args, world, rank, local):
    import torch

    import gpudemod as G
    from gpudemod import synth
    from oracle import oracle as O
    dev = torch.device("cuda", local)
    n_scene = min(max(32, 2 * (args.warmup + args.steps)), 96)
    scene, specs = synth.mixed_scene(device=dev, block=BLOCK, seed=synth.CONFIG_SEEDS[2] + rank)
    blocks = torch.empty((n_scene, BLOCK), dtype=torch.complex64, device=dev)
    for b in range(n_scene):
        blocks[b] = scene.next_block()
    torch.cuda.synchronize()
    mode = {"NFM": G.MODE_NFM, "AM": G.MODE_AM, "USB": G.MODE_USB, "LSB": G.MODE_LSB, "CW": G.MODE_CW}
    chans = []
    for kind, off in specs:
        out_rate, taps, bw = synth.MODE_TABLE[kind]
        chans.append(dict(kind=kind, T=taps, D=FS // out_rate, out_rate=out_rate, bw=bw, off=off))

    # extraction forms per (taps, decimation) class chosen by the autotuner,
    # measured on this GPU before anything is timed
    tune = None
    if not args.no_autotune:
        from gpudemod import autotune
        classes = sorted({(c["T"], c["D"]) for c in chans})
        table, report = autotune.tune(FS, BLOCK, classes)
        names = {G.FORM_DENSE: "dense", G.FORM_WIDE: "wide", G.FORM_GROUP: "group", G.FORM_MOD: "mod"}
        tune = {"table": table,
                "chosen": {f"T{T}_D{D}": f"{names[f]}" + (f"/pg{pg}" if pg else "") for T, D, f, pg in table},
                "candidates_ms": {f"T{T}_D{D}": {names[f] + (f"/pg{pg}" if pg else ""): round(ms, 4)
                                                 for (f, pg), ms in times.items()}
                                  for (T, D), times in report.items()}}

    def make_runner():
        r = G.ChannelRunner(FS, BLOCK, max_channels=128, max_taps=1024)
        if tune is not None:
            r.set_autotune_table(tune["table"])
        for i, c in enumerate(chans):
            r.admit(i, c["off"], c["bw"], c["out_rate"], c["T"], mode[c["kind"]], G.CH_AUDIO48K)
        return r

    def cpu_baseline(blocks):
        omode = {"NFM": O.MODE_NFM, "AM": O.MODE_AM, "USB": O.MODE_USB, "LSB": O.MODE_LSB, "CW": O.MODE_CW}
        oc = [CpuChannel(O, FS, c["off"], c["bw"], c["out_rate"], c["T"], omode[c["kind"]], c["kind"], False)
              for c in chans]
        nb = args.cpu_blocks
        bnp = [blocks[b].cpu().numpy() for b in range(nb)]
        threads = host_threads()

        def work(c):
            for b in range(nb):
                c.process(bnp[b])

        t0 = time.perf_counter()
        with cf.ThreadPoolExecutor(max_workers=threads) as ex:
            list(ex.map(work, oc))
        dt = time.perf_counter() - t0
        return {"value": len(oc) * nb * BLOCK / dt / 1e6, "unit": "channel-MS/s", "cores": threads, "kind": "port",
                "sample": f"{len(oc)} channels x {nb} blocks of 2^20 through the oracle chain ({dt:.1f} s wall)"}

    runner = make_runner()
    form_key = {G.FORM_DENSE: "extract_dense", G.FORM_WIDE: "extract_wide", G.FORM_GROUP: "extract_group",
                G.FORM_MOD: "extract_mod"}
    for i, c in enumerate(chans):  # the runner's own form per channel (slots in admission order)
        c["form"] = form_key[runner.channel_form(i)[0]]
    res = measure_batch(args, world, rank, local, runner, blocks, n_scene, chans, "mixed", make_runner,
                        cpu_baseline)
    runner.close()
    if res is None:
        return None
    line = {"metric": "aggregate channel-MS/s on 1 B200, mixed-mode uneven batch", "unit": "channel-MS/s"}
    line.update(res)
    if tune is not None:
        line["autotune"] = {k: v for k, v in tune.items() if k != "table"}
    line["config"] = {"workload": MIXED_WORKLOAD, "channels": len(chans), "block": BLOCK,
                      "inputs": f"{n_scene} consecutive 8 MiB blocks resident in HBM ({n_scene * 8} MiB > L2)",
                      "parallelism": f"channel shards, {world} GPU(s), no data-path collective"}
    return line


SERVE_BLOCK = 262144
SERVE_WORKLOAD = ("Serving stream: continuous seeded 10 MS/s cf32 (12 WFM + 48 narrow stations, AWGN), blocks "
                  "of 262144; demod requests Poisson (lambda 50/s, and 200/s to saturate the 512-channel cap), "
                  "uniform-random frequency, modes WFM .30 (stereo + RDS) / NFM .30 / AM .20 / SSB .15 / CW .05, "
                  "lifetimes log-uniform 0.1-30 s, cap 512, admission by a device-memory budget")


def serve_phases(args, world, rank, local, seconds):
    """The serving stream at lambda = 50/s (the serving config) and at
    200/s (holding the 512-channel cap), `seconds` of stream each.  Requests
    join and leave at block boundaries; each block is submitted from pinned
    host memory and runs every live channel.  Per block: device latency = the
    runner's event time from submit to outputs in host memory; wall = host
    boundary (retire/admit) + submit + wait, by the host clock.  At the end,
    the plain per-signal runner on the saturated phase's final population."""
    import torch

    import gpudemod as G
    from gpudemod import serving as SV
    from gpudemod import synth
    dev = torch.device("cuda", local)
    period = SERVE_BLOCK / FS
    n_blocks = max(16, int(seconds / period))
    phases = [("c3", 50.0), ("saturated", 200.0)]
    scene, _ = synth.serving_scene(device=dev, block=SERVE_BLOCK, seconds=len(phases) * n_blocks * period + 1,
                                   seed=synth.CONFIG_SEEDS[3] + rank)
    pinned = []
    for _ in range(len(phases) * n_blocks):
        pinned.append(scene.next_block().cpu().pin_memory())
    torch.cuda.synchronize()
    budget = 6 << 30
    runner = G.ChannelRunner(FS, SERVE_BLOCK, max_channels=512, max_taps=1024, device_mem_budget=budget)
    warm = 8  # blocks after the stream opens (every channel acquiring) left out of the latency figures
    out, live_specs = {}, None
    l0 = G.kernel_launch_count()
    clk = ClockSampler(local).__enter__()
    for pi, (name, lam) in enumerate(phases):
        reqs = SV.poisson_requests(synth.CONFIG_SEEDS[3] + 17 * pi + rank, n_blocks * period, rate_hz=lam)
        loop = SV.ServingLoop(runner, SERVE_BLOCK, FS)
        # close the previous phase's channels: each phase opens at its own steady state
        for slot in list(range(512)):
            try:
                runner.retire(slot)
            except G.GPUDError:
                pass
        reqs.sort(key=lambda q: q.t_arrive)
        qi = 0
        lat, wall, live, adm_ms, used, d2h = [], [], [], [], [], []
        for k in range(n_blocks):
            t_now = k * period
            arr = []
            while qi < len(reqs) and reqs[qi].t_arrive <= t_now:
                arr.append(reqs[qi])
                qi += 1
            h0 = time.perf_counter()
            loop.boundary(t_now, arr)
            h1 = time.perf_counter()
            stt = loop.process(pinned[pi * n_blocks + k])
            h2 = time.perf_counter()
            adm_ms.append((h1 - h0) * 1e3)
            wall.append((h2 - h0) * 1e3)
            lat.append(stt["last_block_ms"])
            live.append(len(loop.live))
            used.append(stt["device_bytes_used"])
            d2h.append(stt["last_d2h_bytes"])
        L = np.array(lat[warm:])
        W = np.array(wall[warm:])
        n_live = np.array(live[warm:])
        out[name] = {
            "lambda_per_s": lam, "blocks": n_blocks, "block_period_ms": period * 1e3,
            "channels_mean": float(n_live.mean()), "channels_max": int(np.max(live)),
            "p50_block_ms": float(np.percentile(L, 50)), "p99_block_ms": float(np.percentile(L, 99)),
            "max_block_ms": float(L.max()),
            "wall_p99_block_ms": float(np.percentile(W, 99)),
            "admitted": loop.admitted, "admission_refusals": loop.rejected, "retired": loop.retired,
            "boundary_host_ms_p99": float(np.percentile(adm_ms[warm:], 99)),
            "device_bytes_used_max": int(max(used)), "device_bytes_budget": budget,
            "throughput_channel_msps": float(n_live.sum() * SERVE_BLOCK / (W.sum() * 1e-3) / 1e6),
            "capacity_channel_msps": float(n_live.sum() * SERVE_BLOCK / (L.sum() * 1e-3) / 1e6),
            "realtime_need_channel_msps": float(n_live.mean() * FS / 1e6),
            "realtime": bool(np.percentile(W, 99) < period * 1e3),
            "d2h_bytes_per_block_mean": float(np.mean(d2h[warm:])),
        }
        live_specs = [SV.channel_spec(q) for _, q in loop.live.values()]
    clk.__exit__(None, None, None)
    launches = G.kernel_launch_count() - l0
    runner.close()
    plain = {"value": None, "unit": "channel-MS/s", "channels": len(live_specs)}
    if rank == 0 and args.plain_steps > 0 and not args.profile_only:
        pr = G.ChannelRunner(FS, SERVE_BLOCK, max_channels=512, max_taps=1024)
        for spec in live_specs:
            pr.admit(*spec)
        pr.set_schedule(G.SCHED_PLAIN)
        pr.process_block(pinned[0])
        t0 = time.perf_counter()
        for s in range(args.plain_steps):
            pr.process_block(pinned[1 + s])
        plain["value"] = len(live_specs) * SERVE_BLOCK * args.plain_steps / (time.perf_counter() - t0) / 1e6
        pr.close()
    del pinned
    return out, plain, launches, clk.summary()


SERVING_DEFINITIONS = ("per block: p50/p99 = device latency (runner events, submit from pinned host memory to "
                       "outputs in host memory); throughput = live channels x block samples / host wall time of "
                       "boundary (retire/admit) + submit + wait; capacity = the same over device latency; plain = "
                       "the per-signal runner (one channel at a time, H2D/D2H per channel) on the saturated "
                       "phase's final population, host wall time")


def serving_summary(out, plain):
    """The serving target's figures: the saturated phase (>= 512 live
    channels) against p99 < 10 ms and >= 5x the plain runner."""
    sat = out["saturated"]
    sp = sat["throughput_channel_msps"] / plain["value"] if plain["value"] else None
    return {"channels_mean": sat["channels_mean"], "channels_max": sat["channels_max"],
            "p50_block_ms": sat["p50_block_ms"], "p99_block_ms": sat["p99_block_ms"],
            "wall_p99_block_ms": sat["wall_p99_block_ms"], "block_period_ms": sat["block_period_ms"],
            "throughput_channel_msps": sat["throughput_channel_msps"],
            "realtime_need_channel_msps": sat["realtime_need_channel_msps"],
            "plain_runner_channel_msps": plain["value"], "speedup_batched_vs_plain": sp,
            "target_met": bool(sat["channels_mean"] >= 512 and sat["p99_block_ms"] < 10.0
                               and sat["wall_p99_block_ms"] < sat["block_period_ms"] and (sp or 0) >= 5.0),
            "c3_lambda50": {k: out["c3"][k] for k in ("channels_mean", "p50_block_ms", "p99_block_ms",
                                                        "throughput_channel_msps")},
            "definitions": SERVING_DEFINITIONS}


def run_serving(args, world, rank, local):
    """The serving workload as its own line."""
    out, plain, launches, clocks = serve_phases(args, world, rank, local, args.serve_seconds)
    if rank != 0:
        return None
    sat = out["saturated"]
    value = world * sat["throughput_channel_msps"]
    return {"metric": "serving: aggregate channel-MS/s at the 512-channel cap; p99 block latency",
            "value": value, "unit": "channel-MS/s", "n_gpus": world, "steps": sat["blocks"], "warmup": 8,
            "ms_per_step": sat["p50_block_ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (f64 NCO/PLL state)",
            "data": "synthetic (seeded stream and request process)",
            "config": {"workload": SERVE_WORKLOAD, "block": SERVE_BLOCK, "max_channels": 512,
                       "parallelism": f"independent request streams, {world} GPU(s)"},
            "e2e": {"value": value, "unit": "channel-MS/s", "h2d_bytes_per_step": SERVE_BLOCK * 8,
                    "d2h_bytes_per_step": sat["d2h_bytes_per_block_mean"],
                    "note": "every block from pinned host memory to outputs in host memory"},
            "serving": out, "serving_target": serving_summary(out, plain),
            "plain_runner": plain, "gpu_launches": launches, "clocks": clocks}


HEADROOM_BLOCK = 1 << 20
HEADROOM_WORKLOAD = ("Headroom stress: continuous seeded 61.44 MS/s cf32 (48 WFM + 160 narrow stations, AWGN) in "
                     "2^20-sample blocks, 2048 concurrent channels (WFM 30 % with stereo + RDS at D 192; NFM / AM / "
                     "SSB / CW at the mixed batch's 40:30:30:20 ratios), FIR lengths uniform 64-1024 taps, "
                     "decimation log-uniform over the exact divisors of 61,440,000 in [16, 2400], churn: Poisson "
                     "200/s channel replacements at block boundaries; audio at the demod rate")


def run_headroom(args, world, rank, local):
    """Headroom stress in serving mode: the population held at 2048 channels,
    each block boundary retires a Poisson(200/s x period) number of random
    channels and admits as many new draws.  value: blocks resident in HBM,
    three in flight, outputs on the device; e2e: each block from pinned host
    memory to outputs in host memory, p50/p99 of the runner's block time."""
    import torch

    import gpudemod as G
    from gpudemod import serving as SV
    from gpudemod import synth
    dev = torch.device("cuda", local)
    fs, blk, n_live = synth.HEADROOM_FS, HEADROOM_BLOCK, args.headroom_channels
    period = blk / fs
    n_val = args.warmup + args.steps
    n_blocks = 2 * n_val
    scene, wfm_offs, narrow = synth.headroom_scene(device=dev, block=blk, seconds=n_blocks * period + 1,
                                                   seed=synth.CONFIG_SEEDS[4] + rank)
    blocks = torch.empty((n_blocks, blk), dtype=torch.complex64, device=dev)
    for b in range(n_blocks):
        blocks[b] = scene.next_block()
    torch.cuda.synchronize()
    mix = SV.HeadroomMix(synth.CONFIG_SEEDS[4] + 101 * rank, wfm_offs, narrow)
    churn = np.random.default_rng(synth.CONFIG_SEEDS[4] + 7 + rank)
    # spare slots: a retired slot is reused only after the blocks in flight that
    # still read it have completed
    runner = G.ChannelRunner(fs, blk, max_channels=n_live + 64, max_taps=1024, device_mem_budget=48 << 30)
    live = {}

    def admit(req):
        live[req.rid] = (runner.admit(*SV.channel_spec(req)), req)

    def boundary():
        k = int(churn.poisson(200.0 * period))
        for rid in churn.choice(sorted(live), size=min(k, len(live)), replace=False):
            slot, _ = live.pop(int(rid))
            runner.retire(slot)
        while len(live) < n_live:
            admit(mix.draw())
        return k

    def chan_dicts():
        return [dict(kind=q.kind, T=q.taps, D=fs // q.out_rate, out_rate=q.out_rate, pcm=False)
                for _, q in live.values()]

    for _ in range(n_live):
        admit(mix.draw())
    stream = torch.cuda.ExternalStream(runner.stream_handle(), device=dev)
    # the e2e pass's blocks in pinned host memory, prepared before any timing
    pinned = [blocks[n_val + b].cpu().pin_memory() for b in range(n_val)]

    # ---- value: blocks in HBM, three in flight, outputs on the device -------
    runner.set_host_outputs(False)
    runner.set_profiling(True)
    clk = ClockSampler(local).__enter__()
    pipelined(runner, [blocks[b] for b in range(args.warmup)])
    runner.reset_stats()
    l0 = G.kernel_launch_count()
    stage_acc, flop, ch_samples, churned = {}, 0.0, 0, 0
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    tickets = []
    for s in range(args.steps):
        churned += boundary()
        w = algorithmic_work(chan_dicts(), n_in=blk)
        flop += w["per_block_flop"]
        ch_samples += len(live) * blk
        tickets.append(runner.submit(blocks[args.warmup + s]))
        if len(tickets) >= 3:
            runner.wait(tickets[-3])
            for name, ms in runner.stage_times():
                stage_acc.setdefault(name, []).append(ms)
    runner.wait(tickets[-1])
    for name, ms in runner.stage_times():
        stage_acc.setdefault(name, []).append(ms)
    e1.record(stream)
    torch.cuda.synchronize()
    launches = G.kernel_launch_count() - l0
    t_ms = max_over_ranks(world, e0.elapsed_time(e1))
    value = world * ch_samples / (t_ms * 1e-3) / 1e6
    st_value = runner.stats()

    # ---- e2e: pinned host memory in, outputs in host memory, per block ------
    runner.set_profiling(False)
    runner.set_host_outputs(True)
    for b in range(args.warmup):
        boundary()
        runner.process_block(pinned[b])
    lat, d2h, used, e2e_samples = [], [], [], 0
    barrier(world)
    for s in range(args.steps):
        boundary()
        runner.process_block(pinned[args.warmup + s])
        st = runner.stats()
        lat.append(st["last_block_ms"])
        d2h.append(st["last_d2h_bytes"])
        used.append(st["device_bytes_used"])
        e2e_samples += len(live) * blk
    clk.__exit__(None, None, None)
    L = np.array(lat)
    busy_ms = max_over_ranks(world, float(L.sum()))
    e2e = world * e2e_samples / (busy_ms * 1e-3) / 1e6
    hist = {}
    for _, q in live.values():
        hist[q.kind] = hist.get(q.kind, 0) + 1
    runner.close()
    if rank != 0:
        return None

    # ---- roofline: the whole block, and the dominant kernel ------------------
    hbm_peak, peak_kind = measured_peaks()
    fp32, _ = fp32_fma_peak()
    kern = {k: statistics.mean(v) for k, v in stage_acc.items()
            if k not in ("h2d", "d2h") and not k.startswith("wait")}
    block_ms = t_ms / args.steps
    work = algorithmic_work(chan_dicts(), n_in=blk)
    b_min = sum(v["bytes"] for k, v in work.items() if isinstance(v, dict) and not k.startswith("extract_"))
    t_roof = max(flop / args.steps / (fp32 * 1e12), b_min / (hbm_peak * 1e9)) * 1e3
    dom = max(kern, key=kern.get)
    dk = stage_key(dom)
    wdk = work.get(dk, {"flop": 0})
    ach = wdk["flop"] / (kern[dom] * 1e-3) / 1e12
    roof = {"bound": "fp32", "achieved": ach, "peak": fp32, "unit": "TFLOP/s", "frac": ach / fp32,
            "peak_source": "FP32 FMA microbenchmark, measured in this run", "kernel": dom,
            "ms_per_launch": kern[dom], "algorithmic_flop": wdk["flop"],
            "traffic": NCU_TRAFFIC_HEADROOM_512.get(dk) if n_live == 512 else None,
            "traffic_at_512_channels": NCU_TRAFFIC_HEADROOM_512.get(dk),
            "block": {"gflop": flop / args.steps / 1e9, "min_bytes": b_min, "roofline_ms": t_roof,
                      "measured_ms": block_ms, "frac": t_roof / block_ms,
                      "hbm_peak_gbs": hbm_peak, "hbm_peak_source": peak_kind}}
    cpu = None
    if not args.no_cpu and not args.profile_only:
        from oracle import oracle as O
        omode = {"WFM": O.MODE_WFM_STEREO, "NFM": O.MODE_NFM, "AM": O.MODE_AM, "USB": O.MODE_USB,
                 "LSB": O.MODE_LSB, "CW": O.MODE_CW}
        sample = [q for _, q in list(live.values())[:128]]
        x = blocks[0].cpu().numpy()

        def work1(q):
            out_rate, taps, bw = synth.MODE_TABLE[q.kind]
            O.OracleChannel(fs, q.offset_hz, bw, q.out_rate, q.taps, omode[q.kind], rds=q.kind == "WFM").process(x)

        threads = host_threads()
        t0 = time.perf_counter()
        with cf.ThreadPoolExecutor(max_workers=threads) as ex:
            list(ex.map(work1, sample))
        dt = time.perf_counter() - t0
        cpu = {"value": len(sample) * blk / dt / 1e6, "unit": "channel-MS/s", "cores": threads, "kind": "port",
               "sample": f"{len(sample)} channels of the mix x 1 block of 2^20 through the oracle chain "
                         f"({dt:.1f} s wall)"}
    return {
        "metric": "headroom stress: aggregate channel-MS/s at 2048 channels with churn; fraction of the "
                  "FP32/HBM roofline", "unit": "channel-MS/s",
        "value": value, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": block_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (f64 NCO/PLL state)", "data": "synthetic (seeded stream and channel draws)",
        "config": {"workload": HEADROOM_WORKLOAD, "channels": n_live, "block": blk, "sample_rate": fs,
                   "mix_at_end": hist, "churned_per_pass": churned,
                   "inputs": f"{n_blocks} consecutive 8 MiB blocks resident in HBM ({n_blocks * 8} MiB > L2)",
                   "parallelism": f"channel shards, {world} GPU(s), no data-path collective"},
        "e2e": {"value": e2e, "unit": "channel-MS/s", "h2d_bytes_per_step": blk * 8,
                "d2h_bytes_per_step": float(np.mean(d2h)), "p50_block_ms": float(np.percentile(L, 50)),
                "p99_block_ms": float(np.percentile(L, 99)), "max_block_ms": float(L.max())},
        "latency_ms": {"p50": st_value["p50_block_ms"], "p99": st_value["p99_block_ms"],
                       "block_period_ms": period * 1e3},
        "realtime": {"need_channel_msps": n_live * fs / 1e6,
                     "met": bool(np.percentile(L, 99) < period * 1e3)},
        "device_bytes_used_max": int(max(used)),
        "roofline": roof,
        "stage_ms": {k: round(v, 4) for k, v in sorted(kern.items(), key=lambda kv: -kv[1])},
        "cpu_baseline": cpu,
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }


def plan_only(args, world, rank):
    """The process world and the FM band channel shards, without GPU work:
    rank 0 prints {"n_gpus", "shards"} gathered from every rank."""
    import torch.distributed as dist
    synth = standalone("synth")
    _, stations = synth.fm_band_scene(device="cpu", block=BLOCK, n_stations=N_CH, seconds=1.0,
                                      seed=synth.CONFIG_SEEDS[1])
    mine = [sid for sid, _ in fm_band_shard(stations, world, rank)]
    shards = [None] * world
    if world > 1:
        dist.all_gather_object(shards, mine)
    else:
        shards = [mine]
    if rank == 0:
        print(json.dumps({"n_gpus": world, "channels": N_CH * world, "shards": shards}))


def main():
    args = parse()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(spawn_ranks(args))
    if args.impl == "reference":
        return run_reference(args)
    world, rank, local = dist_setup(args)
    if args.plan_only:
        plan_only(args, world, rank)
    elif args.workload == "serving":
        line = run_serving(args, world, rank, local)
    elif args.workload == "headroom":
        line = run_headroom(args, world, rank, local)
    elif args.workload == "mixed":
        line = run_mixed(args, world, rank, local)
    else:
        line = run_fm_band(args, world, rank, local)
    barrier(world)
    if rank == 0 and not args.plan_only:
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
