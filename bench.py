"""Benchmark: Analyse frame-pairs/s at 1080p (bit-exact vectors) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl svpflow_b200|reference]

Workload (the reference's 1080p configuration): a seeded synthetic 1920x1080 YUV420P8
clip of 240 frames (global motion in [-24,24]^2, 8 moving objects in [-48,48]^2,
noise sigma 2); Super {pel:2} (bilinear sub-pixel planes); Analyse
{block:{w:16,overlap:3},main:{search:{type:3,distance:16,satd:true}}} -- block 16,
overlap 8, UMH radius 16, SATD + chroma, forward and backward vectors. One step = the
hot path over the whole clip: Super over 240 frames, then Analyse of its 240 output
frames (frame n paired with min(n+1, 239)). `value` = frame pairs per second with the
source frames resident in HBM; `e2e` = the same through the host-buffer C ABI call
(host frames in, payloads out, copies inside the timed region).

Multi-GPU: one process per GPU; each rank analyses its own clip (weak scaling, no data
collective); time = max over ranks.
--impl reference times the CPU restatement of the reference (oracle/) on all host
threads over a bounded sample of the same workload.

Other workloads (one JSON line each, same keys):
  --workload batched   64 clips of uneven size and length (resolution from 360p..1440p,
                       16-240 frames log-uniform, block 8 or 16, else the 1080p options)
                       analysed by one persistent launch replayed from a CUDA graph, with the
                       autotuned launch shape; `plain_per_clip` times the same clips through
                       the per-clip path one after another, and every payload is compared.
  --workload 2160p10   a 3840x2160 10-bit clip (uint16 samples) of 120 frames, Super {pel:4},
                       Analyse block 8 / overlap 4 / exhaustive r8 / SATD + chroma; the CPU leg
                       and the parity check use the oracle's uint16 build.
  --workload render    SmoothFps's single-warp render (algorithm 2, no masks) of 32 1080p frames
                       from their pel-2 super frames and vector planes; frames/s, CPU leg = the
                       oracle's render on all host threads, every frame compared. Beside it:
                       algorithm 13 (two sources) and algorithm 21 with its mask planes made
                       from the payloads in the same step, each checked on a few frames.
  --workload served    Poisson arrivals of clips (360p..2160p, 8-600 frames) into the
                       continuous-batching server under an HBM budget, at each --rates value;
                       p50 / p99 per-frame-pair latency (arrival of the clip to its payload in
                       host memory) and aggregate frame-pairs/s.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "open-svpflow_b200"))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from svpflow_b200.shard import clips_of_rank, shard_clip  # noqa: E402
from svpflow_b200.synth import (ANALYSE_OPT, CONFIGS, SUPER_OPT, analyse_opt_for_block, batched_mix,  # noqa: E402
                                 make_clip, make_clip_device, served_stream)

WORKLOAD = "1080p"  # the single-clip workload of a run: "1080p" (default) or "640x360"
METRIC = "Analyse frame-pairs/s at 1080p (bit-exact MVs), batched vs plain; p99 latency"
DESC = {
    "1080p": "1080p YUV420P8 {n}-frame synthetic clip per GPU, Super {s}, Analyse {a} (block 16, overlap 8, "
             "UMH r16, SATD+chroma, fwd+bwd)",
    "640x360": "640x360 YUV420P8 {n}-frame synthetic clip per GPU, Super {s}, Analyse {a} (block 16, overlap 0, "
               "hex2 r2, luma SAD + chroma, fwd+bwd)",
}
UNIT = "frame-pairs/s"
# DRAM bytes per frame pair of the Analyse launch at 1080p: ncu's dram__bytes_read.sum +
# dram__bytes_write.sum of the three kernels of the 240-pair launch (one-pass counters):
# analyse_kernel 5.55 + 0.77 GB, analyse_level0_kernel 16.17 + 0.40 GB, analyse_finish_kernel
# 0.14 + 0.08 GB (profiles/analyse_1080p_240_counters.md)
TRAFFIC_PER_PAIR = 23.11e9 / 240
# DRAM bytes of one 1080p render launch with the 8 x 8 effective block (ncu capture: 4.13 MB read,
# the written frame stays in L2)
RENDER_TRAFFIC_PER_FRAME = 4.14e6
# graph replays per timed render step (about 40 ms, so the clock sampler sees the step)
RENDER_REPLAYS = 48
# int32 lanes per SM on sm_100 (64 on the ALU pipe, 64 IMAD on the FMA-heavy pipe; ncu's pipe counters
# of the Analyse kernel put the ALU pipe's peak at 2 warp instructions per SM cycle) and the SM clock
# ceiling, for the nominal integer peak
INT32_LANES_PER_SM = 128
# integer ops per frame pair (oracle counts of the workloads' compares), when the CPU leg is skipped
OPS_PER_PAIR = {"1080p": 19.38e9}
# why the Analyse launch reaches the fraction it does, from the ncu counters of the 240-pair launch
# in profiles/analyse_1080p_240_counters.md: issue utilisation (warp instructions / (4 schedulers x
# SMs x the launch's SM cycles)) x useful lane fraction (algorithmic ops / executed lane slots)
ROOF_DECOMPOSITION = {"issue_active": 0.341, "useful_lane_fraction": 0.332,
                      "source": "ncu counters of the 240-pair 1080p launch (analyse_kernel 142.9 G + "
                                "analyse_level0_kernel 295.0 G + analyse_finish_kernel 0.03 G warp instructions "
                                "in 1105.5 ms): 1.82 G warp instructions = 58.4 G lane slots per pair for 19.4 G "
                                "algorithmic ops (profiles/analyse_1080p_240_counters.md)"}
# the CPU legs time this many frame pairs per host thread, so that their figure is a throughput
# (dynamic scheduling over many pairs) rather than the latency of the slowest pair
CPU_PAIRS_PER_THREAD = 4
# the batched object of the default line runs this launch shape (the one svpf_batch_autotune picks
# for the 64-clip mix), so the default run spends no time on autotune trials
BATCH_SHAPE = "nt32_b8:8"
# the served object's arrival rates, clips/s: below the server's capacity, and the configuration's lowest
SERVED_RATES = "0.25,5"
SM_MAX_MHZ = 1965.0


def _sm_count() -> int:
    import torch

    return torch.cuda.get_device_properties(0).multi_processor_count


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _chain(an, nf: int, a_ms: float) -> dict:
    """The non-roofline bound: every pair of a launch runs concurrently (one CTA each), so the launch
    lasts about one pair's serial block chain; per level-0 block of one direction."""
    vd = an.vector_header()
    sms = _sm_count()
    waves = -(-nf // (3 * sms)) if nf > 2 * sms else 1  # 3-CTA shape above 2 pairs per SM, else one wave
    l0 = vd[11] * vd[12]
    return {"pairs_in_flight": min(nf, 3 * sms if nf > 2 * sms else nf), "waves": waves,
            "pair_latency_ms": a_ms / waves, "level0_blocks_per_direction": l0,
            "us_per_level0_block": a_ms / waves * 1000.0 / max(l0, 1),
            "note": "blocks of a level run in the reference's serial order (each reads its processed "
                    "neighbours); the time per block, not issue or memory throughput, bounds one pair"}


def _config(nframes: int, world: int, shard_frames: bool = False) -> dict:
    c = CONFIGS[WORKLOAD]
    return {
        "workload": DESC[WORKLOAD].format(n=nframes, s=SUPER_OPT[WORKLOAD], a=ANALYSE_OPT[WORKLOAD]),
        "width": c["width"], "height": c["height"],
        "frames_per_gpu": -(-nframes // world) if shard_frames else nframes,
        "pairs_per_step": nframes if shard_frames else nframes * world,
        "l2": ("inputs larger than L2 (240 super frames = 3.7 GB per GPU)" if WORKLOAD == "1080p" else
               "inputs smaller than L2: a 256 MB write flushes L2 before every step, outside the timed events"),
        "parallelism": ((f"dp{world}: one clip split into contiguous frame ranges (svpflow_b200.shard), no collective"
                         if shard_frames else f"dp{world}: a clip per GPU, no collective")
                        if world > 1 else "single GPU"),
    }


class ClockSampler:
    """nvidia-smi clock / throttle samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.gpu_id, f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
            t0 = time.time()  # nvidia-smi takes a moment to start: let its first sample land first
            while not self.lines and time.time() - t0 < 3.0 and self.proc.poll() is None:
                time.sleep(0.02)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"), p[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def _gpu_id(torch, dev: int) -> str:
    try:
        u = str(torch.cuda.get_device_properties(dev).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        return str(dev)


_CPU_CLIPS = {}


def cpu_reference(nframes_total: int, threads: int, pairs: int, seed: int = 1000):
    """Times the oracle (CPU restatement of the reference) on `pairs` output frames of the
    workload: Super over the frames they need, then Analyse, on `threads` host threads.
    The clip (frames 0..pairs of the seeded workload clip) is made once per seed."""
    from oracle import oracle as orc

    c = CONFIGS[WORKLOAD]
    w, h = c["width"], c["height"]
    n = pairs + 1
    key = (WORKLOAD, n, seed)
    if key not in _CPU_CLIPS:
        _CPU_CLIPS[key] = make_clip(w, h, n, seed=seed, motion=c["motion"], objects=c["objects"],
                                    object_motion=c["object_motion"])
    clip = _CPU_CLIPS[key]
    so = orc.super_opts(w, h, SUPER_OPT[WORKLOAD])
    ao = orc.analyse_opts(orc.sdata(so), ANALYSE_OPT[WORKLOAD], None, w, h)
    orc.total_counters(reset=True)
    t0 = time.perf_counter()
    supers = orc.build_super_many(so, clip, threads)
    pay = orc.analyse_clip(ao, so, supers, 0, pairs, threads)
    dt = time.perf_counter() - t0
    cpu_reference.counters = orc.total_counters(reset=True)  # the sample's compares (instrumentation)
    return dt, pay, clip


def _cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def _spread(v) -> dict:
    """Mean, min, max and relative standard deviation of per-step figures."""
    m = statistics.mean(v)
    return {"mean": m, "min": min(v), "max": max(v), "n": len(v),
            "rel_stdev": (statistics.stdev(v) / m) if len(v) > 1 and m else 0.0}


def _one_core(pairs: int = 2) -> dict:
    """The same oracle on one host thread over `pairs` output frames (the per-core figure)."""
    dt, _, _ = cpu_reference(240, 1, pairs, seed=1999)
    return {"value": pairs / dt, "unit": UNIT, "cores": 1, "sample": f"{pairs} output frames, 1 thread"}


def run_reference(args, rank: int):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    pairs = min(max(args.cpu_pairs or CPU_PAIRS_PER_THREAD * threads, 2), 239)
    times = []
    for i in range(args.warmup + args.steps):
        dt, _, _ = cpu_reference(240, threads, pairs, seed=1000)
        if i >= args.warmup:
            times.append(dt)
    total = sum(times)
    value = pairs * args.steps / total
    sample = (f"output frames 0..{pairs - 1} of the seeded 1080p clip (Super + Analyse) per step, "
              f"{pairs / threads:.1f} frame pairs per host thread on {threads} threads (throughput, not one "
              f"pair's latency); oracle/ C restatement of the reference (the Rust reference cannot be built here)")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": _config(240, 1),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample,
                         "cpu_model": _cpu_model(), "one_core": _one_core(),
                         "step_pairs_per_s": _spread([pairs / t for t in times])},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


class _DevBytes:
    """A device byte range as a torch tensor (CUDA array interface; no copy)."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "|u1", "data": (ptr, False), "version": 3}


def _init_dist(world, local):
    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=900))
    return torch, dist


def _max_over_ranks(torch, dist, world, v: float, dev) -> float:
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_render(args, world: int, rank: int, local: int):
    """SmoothFps's single-warp render (algorithm 2, interpolated motion, no masks) of 1080p frames on
    the device: sources are the clip's pel-2 super frames, motion the vector planes of its own Analyse
    payloads (both made on the device first, untimed). One step renders every frame's three planes;
    `value` = frames/s. The CPU leg runs the oracle's render on the same frames, all host threads."""
    torch, dist = _init_dist(world, local)
    import concurrent.futures

    import svpflow_b200 as sv
    from oracle import oracle as orc

    c = CONFIGS["1080p"]
    w, h = c["width"], c["height"]
    nf = args.frames or 32
    dev = torch.device("cuda", local)
    clip = make_clip(w, h, nf + 1, seed=1000 + rank, motion=c["motion"], objects=c["objects"],
                     object_motion=c["object_motion"])
    sb = sv.Super(w, h, SUPER_OPT["1080p"])
    an = sv.Analyse(sb.sdata, ANALYSE_OPT["1080p"], w, h)
    fb, pl = sb.output_len(), an.payload_len()
    frames_d = torch.from_numpy(clip).to(dev)
    sup_d = torch.empty((nf + 1, fb), dtype=torch.uint8, device=dev)
    pay_d = torch.empty((nf, pl), dtype=torch.uint8, device=dev)
    scr_d = torch.empty(an.scratch_bytes(nf), dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    sh = stream.cuda_stream
    sb.build_device(frames_d.data_ptr(), sup_d.data_ptr(), nf + 1, sh)
    an.analyse_clip_device(sup_d.data_ptr(), nf + 1, 0, nf, pay_d.data_ptr(), scr_d.data_ptr(), sh)
    vd = an.vector_header()
    mw, mh = sv.vector_grid(vd)
    planes = torch.empty((nf, 4 * mw * mh), dtype=torch.int16, device=dev)
    status = torch.zeros(nf, dtype=torch.int32, device=dev)
    sv.vector_planes_device(vd, pay_d.data_ptr(), pl, nf, w, h, planes.data_ptr(), status.data_ptr(), stream=sh)
    del scr_d
    torch.cuda.synchronize()
    hs = sb.super_height
    offs = [0, w * hs, w * hs + (w // 2) * (hs // 2)]
    lens = [w * hs, (w // 2) * (hs // 2), (w // 2) * (hs // 2)]
    strides = [w, w // 2, w // 2]
    # SmoothFps's render configuration: the effective block (block - overlap), origin at half the block
    cfg = dict(width=w, height=h, block_w=vd[2] - vd[9], block_h=vd[3] - vd[10], origin_x=vd[2] // 2,
               origin_y=vd[3] // 2, grid_w=mw, grid_h=mh, source_step=2)
    thr = 128
    out_d = torch.empty((nf, w * h * 3 // 2), dtype=torch.uint8, device=dev)
    dst_offs = [0, w * h, w * h + (w // 2) * (h // 2)]

    def render(f, src_base, mot_base, dst_base, st):
        sv.render_warp_device(cfg, thr, False, True, [src_base + o for o in offs], strides, lens, 1, mot_base,
                              mot_base + mw * mh * 2, [dst_base + o for o in dst_offs], strides, st)

    def step(st):
        for f in range(nf):
            render(f, sup_d[f].data_ptr(), planes[f].data_ptr(), out_d[f].data_ptr(), st)

    for _ in range(args.warmup):
        step(sh)
    torch.cuda.synchronize()
    # one render per frame is a short kernel: the step's launches go into a CUDA graph, replayed
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        step(torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    reps = RENDER_REPLAYS  # a step replays the graph this often, so the clock samples land inside the timing
    with ClockSampler(_gpu_id(torch, local)) as clk:
        for e0, e1 in evs:
            flush.fill_(1)  # inputs partly below L2 size: flush between steps, outside the events
            e0.record(stream)
            for _ in range(reps):
                graph.replay()
            e1.record(stream)
        torch.cuda.synchronize()
    launches = nf * reps * args.steps  # one render_kernel per frame in every replay
    ms = sum(e0.elapsed_time(e1) for e0, e1 in evs)
    # the two-source blend (algorithm 13) on the same frames as SmoothFps feeds it: frame f's and
    # f+1's super frames, the two vector sets of frame f's payload
    blend_d = torch.empty_like(out_d)

    def blend(f, st):
        m0 = planes[f].data_ptr()
        m1 = planes[f].data_ptr() + 2 * mw * mh * 2
        sv.render_blend_device(cfg, thr, True, True, False, [sup_d[f].data_ptr() + o for o in offs], strides, lens,
                               [sup_d[f + 1].data_ptr() + o for o in offs], strides, lens, 1, (m0, m0 + mw * mh * 2),
                               (m1, m1 + mw * mh * 2), [blend_d[f].data_ptr() + o for o in dst_offs], strides, stream=st)

    for f in range(nf):
        blend(f, sh)
    torch.cuda.synchronize()
    bgraph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(bgraph):
        cs = torch.cuda.current_stream().cuda_stream
        for f in range(nf):
            blend(f, cs)
    torch.cuda.synchronize()
    bms = []
    for _ in range(args.steps):
        flush.fill_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        bgraph.replay()
        e1.record(stream)
        torch.cuda.synchronize()
        bms.append(e0.elapsed_time(e1))
    blend_value = nf / (statistics.mean(bms) / 1000.0)
    # algorithm 21 as SmoothFps runs it from the payloads: the mask planes of all payloads (mask.cover
    # 100, mask.area 100 -> area scale 0.01) and the masked render of frames f and f+1 with the
    # coverage masks and the max magnitude mask as the final one
    ascale = 0.01
    masks_d = torch.empty((nf, 5 * mw * mh), dtype=torch.uint8, device=dev)
    mscr = torch.empty(sv.render_masks_scratch(vd, nf), dtype=torch.uint8, device=dev)
    mstat = torch.zeros(nf, dtype=torch.int32, device=dev)
    masked_d = torch.empty_like(out_d)
    nm = mw * mh

    def masked_step(st):
        sv.render_masks_device(vd, pay_d.data_ptr(), pl, nf, thr, masks_d.data_ptr(), mscr.data_ptr(),
                               mstat.data_ptr(), cover=100, area_scale=ascale, stream=st)
        for f in range(nf):
            m0, m1, mk = planes[f].data_ptr(), planes[f].data_ptr() + 4 * nm, masks_d[f].data_ptr()
            sv.render_masked_device(cfg, thr, ascale, False, True, [sup_d[f].data_ptr() + o for o in offs], strides,
                                    lens, [sup_d[f + 1].data_ptr() + o for o in offs], strides, lens, 1,
                                    (m0, m0 + 2 * nm), (m1, m1 + 2 * nm), (mk, mk + nm), mk + 4 * nm,
                                    [masked_d[f].data_ptr() + o for o in dst_offs], strides, stream=st)

    masked_step(sh)
    torch.cuda.synchronize()
    mgraph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(mgraph):
        masked_step(torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    mms, kms = [], []
    for _ in range(args.steps):
        flush.fill_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        mgraph.replay()
        e1.record(stream)
        torch.cuda.synchronize()
        mms.append(e0.elapsed_time(e1))
        flush.fill_(1)  # the mask planes alone, for the split
        e0.record(stream)
        sv.render_masks_device(vd, pay_d.data_ptr(), pl, nf, thr, masks_d.data_ptr(), mscr.data_ptr(),
                               mstat.data_ptr(), cover=100, area_scale=ascale, stream=sh)
        e1.record(stream)
        torch.cuda.synchronize()
        kms.append(e0.elapsed_time(e1))
    masked_value = nf / (statistics.mean(mms) / 1000.0)
    masks_us_per_payload = statistics.mean(kms) * 1000.0 / nf
    # algorithm 23 as SmoothFps feeds it (frames 1..nf-2): frame f's two sets, the next payload's
    # previous set and the previous payload's current set, the coverage masks of frame f and the max
    # magnitude mask, on the mask planes made above
    m23_d = torch.empty_like(out_d)

    def m23_frame(f, st):
        pl_ = [planes[k].data_ptr() for k in (f - 1, f, f + 1)]
        sets = [(pl_[1], pl_[1] + 2 * nm), (pl_[1] + 4 * nm, pl_[1] + 6 * nm), (pl_[2], pl_[2] + 2 * nm),
                (pl_[0] + 4 * nm, pl_[0] + 6 * nm)]
        mk = masks_d[f].data_ptr()
        sv.render_mode23_device(cfg, thr, True, [sup_d[f].data_ptr() + o for o in offs], strides, lens,
                                [sup_d[f + 1].data_ptr() + o for o in offs], strides, lens, 1, sets, (mk, mk + nm),
                                mk + 4 * nm, [m23_d[f].data_ptr() + o for o in dst_offs], strides, stream=st)

    for f in range(1, nf - 1):
        m23_frame(f, sh)
    torch.cuda.synchronize()
    m23_graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(m23_graph):
        cs = torch.cuda.current_stream().cuda_stream
        for f in range(1, nf - 1):
            m23_frame(f, cs)
    torch.cuda.synchronize()
    m23_ms = []
    for _ in range(args.steps):
        flush.fill_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        m23_graph.replay()
        e1.record(stream)
        torch.cuda.synchronize()
        m23_ms.append(e0.elapsed_time(e1))
    m23_value = (nf - 2) / (statistics.mean(m23_ms) / 1000.0)
    # the scene class of every payload (one launch), timed the same way
    scls = torch.empty(nf, dtype=torch.int32, device=dev)
    sstat = torch.empty(nf, dtype=torch.int32, device=dev)
    sv.scene_class_device(vd, pay_d.data_ptr(), pl, nf, scls.data_ptr(), sstat.data_ptr(), stream=sh)
    sms_ = []
    for _ in range(args.steps):
        flush.fill_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sv.scene_class_device(vd, pay_d.data_ptr(), pl, nf, scls.data_ptr(), sstat.data_ptr(), stream=sh)
        e1.record(stream)
        torch.cuda.synchronize()
        sms_.append(e0.elapsed_time(e1))
    scene_us_per_payload = statistics.mean(sms_) * 1000.0 / nf
    ms_max = _max_over_ranks(torch, dist, world, ms, dev)
    value = nf * reps * world * args.steps / (ms_max / 1000.0)
    # end to end: host super frames and motion planes in, rendered frames out, per step
    sup_h = torch.empty((nf, fb), dtype=torch.uint8).pin_memory()
    sup_h.copy_(sup_d[:nf])
    mot_h = torch.empty_like(planes, device="cpu").pin_memory()
    mot_h.copy_(planes)
    out_h = torch.empty((nf, w * h * 3 // 2), dtype=torch.uint8).pin_memory()
    sup_s = torch.empty((2, fb), dtype=torch.uint8, device=dev)
    mot_s = torch.empty((2, planes.shape[1]), dtype=torch.int16, device=dev)
    out_s = torch.empty((2, w * h * 3 // 2), dtype=torch.uint8, device=dev)

    def e2e_step():
        for f in range(nf):
            k = f & 1
            sup_s[k].copy_(sup_h[f], non_blocking=True)
            mot_s[k].copy_(mot_h[f], non_blocking=True)
            render(f, sup_s[k].data_ptr(), mot_s[k].data_ptr(), out_s[k].data_ptr(), sh)
            out_h[f].copy_(out_s[k], non_blocking=True)
        torch.cuda.synchronize()

    e2e_step()
    t0 = time.perf_counter()
    for _ in range(max(args.e2e_steps, 1)):
        e2e_step()
    e2e_s = _max_over_ranks(torch, dist, world, time.perf_counter() - t0, dev)
    e2e_value = nf * world * max(args.e2e_steps, 1) / e2e_s
    same = bool(torch.equal(out_h.to(dev), out_d))
    line = None
    if rank == 0:
        out_np = out_d.cpu().numpy()
        sup_np = sup_d[:nf].cpu().numpy()
        mot_np = planes.cpu().numpy().view(np.uint16).reshape(nf, 4, mh * mw)
        _, lut = orc.render_luts(thr)
        ocfg = dict(cfg, chroma_y_div=2)

        def cpu_frame(f):
            res = []
            for p in range(3):
                ph = h // (2 if p else 1)
                src = sup_np[f][offs[p]: offs[p] + lens[p]]
                res.append(orc.render_warp_plane(ocfg, p > 0, True, lut, src, strides[p], strides[p] * ph, 1,
                                                 mot_np[f][0], mot_np[f][1], strides[p], ph))
            return res

        blend_np = blend_d.cpu().numpy()

        def cpu_blend(f):
            g = f
            res = []
            for p in range(3):
                ph = h // (2 if p else 1)
                srcs = [sup_np[f][offs[p]: offs[p] + lens[p]], sup_np[f + 1][offs[p]: offs[p] + lens[p]] if f + 1 < nf
                        else sup_d[f + 1].cpu().numpy()[offs[p]: offs[p] + lens[p]]]
                res.append(orc.render_dual_plane(ocfg, p > 0, True, False, 13, thr, srcs, [strides[p]] * 2,
                                                 [strides[p] * ph] * 2, 1, (mot_np[f][0], mot_np[f][1]),
                                                 (mot_np[g][2], mot_np[g][3]), strides[p], ph))
            return res

        masks_np = masks_d.cpu().numpy().reshape(nf, 5, mh, mw)
        pay_np = pay_d.cpu().numpy()
        masked_np = masked_d.cpu().numpy()
        tlimit = orc.render_threshold_limit(thr, ascale)

        def cpu_masked(f):
            g = f
            om = orc.render_masks(vd, pay_np[f], thr, 100, ascale)
            res = []
            for p in range(3):
                ph = h // (2 if p else 1)
                srcs = [sup_np[f][offs[p]: offs[p] + lens[p]], sup_np[f + 1][offs[p]: offs[p] + lens[p]]]
                res.append(orc.render_dual_plane(ocfg, p > 0, True, False, 21, thr, srcs, [strides[p]] * 2,
                                                 [strides[p] * ph] * 2, 1, (mot_np[f][0], mot_np[f][1]),
                                                 (mot_np[g][2], mot_np[g][3]), strides[p], ph, (om[0], om[1]), om[4],
                                                 tlimit))
            return om, res

        masked_ok = True
        t0 = time.perf_counter()
        masked_res = [cpu_masked(f) for f in range(3)]
        masked_cpu = 3 / (time.perf_counter() - t0)
        for f, (om, res) in enumerate(masked_res):
            masked_ok &= bool(np.array_equal(masks_np[f], om)) and bool(
                np.array_equal(np.concatenate([r.reshape(-1) for r in res]), masked_np[f]))
        m23_np = m23_d.cpu().numpy()

        def cpu_m23(f):
            om = orc.render_masks(vd, pay_np[f], thr, 100, ascale)
            res = []
            for p in range(3):
                ph = h // (2 if p else 1)
                srcs = [sup_np[f][offs[p]: offs[p] + lens[p]], sup_np[f + 1][offs[p]: offs[p] + lens[p]]]
                motions = [(mot_np[f][0], mot_np[f][1]), (mot_np[f][2], mot_np[f][3]),
                           (mot_np[f + 1][0], mot_np[f + 1][1]), (mot_np[f - 1][2], mot_np[f - 1][3])]
                res.append(orc.render_mode23_plane(ocfg, p > 0, True, thr, srcs, [strides[p]] * 2,
                                                   [strides[p] * ph] * 2, 1, motions, (om[0], om[1]), om[4],
                                                   strides[p], ph))
            return res

        t0 = time.perf_counter()
        m23_res = [cpu_m23(f) for f in (1, 2)]
        m23_cpu = 2 / (time.perf_counter() - t0)
        m23_check = {"frames_checked": 2, "bit_exact": all(
            np.array_equal(np.concatenate([r.reshape(-1) for r in m23_res[i]]), m23_np[f])
            for i, f in enumerate((1, 2))), "oracle_frames_per_s_one_thread": m23_cpu}
        scls_np = scls.cpu().numpy()
        scene_check = {"payloads_checked": nf, "bit_exact": bool(all(
            int(scls_np[f]) == orc.scene_class(vd, pay_np[f]) for f in range(nf)))}
        masked_check = {"frames_checked": 3, "bit_exact": masked_ok,
                        "oracle_frames_per_s_one_thread": masked_cpu}
        t0 = time.perf_counter()
        blend_res = [cpu_blend(f) for f in range(4)]
        blend_cpu = 4 / (time.perf_counter() - t0)
        blend_check = {"frames_checked": 4, "bit_exact": all(
            np.array_equal(np.concatenate([r.reshape(-1) for r in blend_res[f]]), blend_np[f]) for f in range(4)),
            "oracle_frames_per_s_one_thread": blend_cpu}
        cpu, parity = None, None
        if not args.no_cpu:
            threads = os.cpu_count() or 1
            t0 = time.perf_counter()
            with concurrent.futures.ThreadPoolExecutor(threads) as ex:
                res = list(ex.map(cpu_frame, range(nf)))
            dt = time.perf_counter() - t0
            cpu = {"value": nf / dt, "unit": "frames/s", "cores": threads, "kind": "port",
                   "sample": f"the same {nf} frames, 3 planes each, oracle/ C restatement of renderer.rs's scalar "
                             f"render, one frame per host thread", "cpu_model": _cpu_model()}
            ok = all(np.array_equal(np.concatenate([r.reshape(-1) for r in res[f]]), out_np[f]) for f in range(nf))
            parity = {"frames_checked": nf, "bit_exact": bool(ok)}
        peak, peak_kind = _peaks()
        per_frame = 2 * w * h * 3 // 2 + 2 * mw * mh * 2  # sources read once + frame written + one motion set
        line = {
            "metric": "SmoothFps single-warp render frames/s at 1080p (bit-exact to the oracle)", "value": value,
            "unit": "frames/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u8", "data": "synthetic",
            "config": {"workload": f"1080p, {nf} frames per step, algorithm 2 (render_mode1_or_2 without masks), "
                                   f"interpolated motion, threshold {thr}, sources = pel-2 super frames, motion = "
                                   f"the clip's own vector planes; a step = {reps} CUDA-graph replays of the "
                                   f"{nf} launches", "frames_per_gpu": nf, "frames_per_step": nf * reps,
                       "l2": "a 256 MB write flushes L2 before every step, outside the timed events; the 32 "
                             "frames' super frames (500 MB) exceed L2 within a step"},
            "clocks": clk.summary(),
            "e2e": {"value": e2e_value, "unit": "frames/s", "h2d_bytes_per_step": int(nf * (fb + planes.shape[1] * 2)),
                    "d2h_bytes_per_step": int(nf * w * h * 3 // 2), "api": "svpf_render_warp_device with host copies",
                    "matches_device_path": same},
            "gpu_launches": int(launches),
            "roofline": {"kernel": "render_kernel<0, 0> (single warp)", "bound": "hbm",
                         "achieved": per_frame * nf * reps / (ms / args.steps / 1000) / 1e9, "peak": peak,
                         "unit": "GB/s", "frac": per_frame * nf * reps / (ms / args.steps / 1000) / 1e9 / peak,
                         "traffic": RENDER_TRAFFIC_PER_FRAME * nf * reps,
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch (1080p "
                                           "frame; the output stays in L2), x frames per step",
                         "peak_source": peak_kind, "algorithmic_bytes_per_frame": per_frame,
                         "note": "issue-bound, not HBM-bound: per sample a tile lookup, motion interpolation and "
                                 "an index computation (67 % issue active in the ncu capture)"},
            "cpu_baseline": cpu, "parity_vs_oracle": parity,
            "blend_mode13": {"value": blend_value, "unit": "frames/s", "kernel": "render_kernel<dual>",
                             "how": "svpf_render_blend_device (algorithm 13: frames f and f+1, the two vector sets "
                                    "of frame f's payload), same frames and timing", "parity_vs_oracle": blend_check},
            "masked_mode21": {"value": masked_value, "unit": "frames/s",
                              "mask_planes_us_per_payload": masks_us_per_payload,
                              "how": f"svpf_render_masks_device for the {nf} payloads (phase {thr}, cover 100, area "
                                     f"scale {ascale}) + svpf_render_masked_device per frame (algorithm 21, final "
                                     "mask = max magnitude), one CUDA-graph replay per step, same timing",
                              "parity_vs_oracle": masked_check},
            "mode23": {"value": m23_value, "unit": "frames/s",
                       "how": f"svpf_render_mode23_device for frames 1..{nf - 2} (frame f's sets, the next "
                              "payload's previous set, the previous payload's current set; frame f's coverage "
                              "masks and max magnitude mask), one CUDA-graph replay per step, same timing",
                       "parity_vs_oracle": m23_check},
            "scene_class": {"us_per_payload": scene_us_per_payload, "how": f"svpf_scene_class_device over the {nf} "
                            "payloads, one launch, CUDA events, L2 flushed before", "parity_vs_oracle": scene_check},
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_2160p10(args, world: int, rank: int, local: int):
    """Config 3: one 2160p 10-bit clip per GPU (uint16 samples 0..1023), Super {pel:4}, Analyse
    block 8 / overlap 4 / exhaustive radius 8 / SATD + chroma. The reference is 8-bit only, so
    the CPU leg is the oracle's uint16 build, and parity is against it."""
    torch, dist = _init_dist(world, local)
    import svpflow_b200 as sv
    from oracle import oracle as orc

    wl = "2160p10"
    c = CONFIGS[wl]
    w, h = c["width"], c["height"]
    nf = args.frames or c["frames"]
    dev = torch.device("cuda", local)
    t0 = time.perf_counter()
    frames_d = make_clip_device(w, h, nf, seed=3000 + rank, motion=c["motion"], objects=c["objects"],
                                object_motion=c["object_motion"], noise=c["noise"], device=dev, bits=c["bits"])
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t0
    sb = sv.Super(w, h, SUPER_OPT[wl], bits=c["bits"])
    an = sv.Analyse(sb.sdata, ANALYSE_OPT[wl], w, h, bits=c["bits"])
    fb, pl = sb.output_len(), an.payload_len()
    supers_d = torch.empty((nf, fb), dtype=torch.uint8, device=dev)
    pay_d = torch.empty((nf, pl), dtype=torch.uint8, device=dev)
    scratch_d = torch.empty(an.scratch_bytes(nf), dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    sh = stream.cuda_stream

    def step(ev=None):
        if ev:
            ev[0].record(stream)
        sb.build_device(frames_d.data_ptr(), supers_d.data_ptr(), nf, sh)
        if ev:
            ev[1].record(stream)
        an.analyse_clip_device(supers_d.data_ptr(), nf, 0, nf, pay_d.data_ptr(), scratch_d.data_ptr(), sh)
        if ev:
            ev[2].record(stream)

    for _ in range(args.warmup):
        step()
    sv.Analyser.device_status(scratch_d.data_ptr(), sh)
    torch.cuda.synchronize()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sv.reset_kernel_launches()
    with ClockSampler(_gpu_id(torch, local)) as clk:
        start.record(stream)
        for i in range(args.steps):
            step(evs[i])
        stop.record(stream)
        torch.cuda.synchronize()
    launches = sv.kernel_launches()
    sv.Analyser.device_status(scratch_d.data_ptr(), sh)
    ms_max = _max_over_ranks(torch, dist, world, start.elapsed_time(stop), dev)
    value = nf * world * args.steps / (ms_max / 1000.0)
    super_ms = statistics.mean(e[0].elapsed_time(e[1]) for e in evs)
    a_ms = statistics.mean(e[1].elapsed_time(e[2]) for e in evs)
    pay_host = pay_d.cpu().numpy()
    # end to end through the host-buffer call; the device-path buffers are released first
    host_frames = frames_d.cpu().pin_memory().numpy().view(np.uint16)
    del supers_d, scratch_d, pay_d, frames_d
    torch.cuda.empty_cache()
    out_host = torch.empty((nf, pl), dtype=torch.uint8).pin_memory().numpy()
    e2e_value, same = None, None
    if args.e2e_steps > 0:
        def e2e_step():
            rc = sv.lib().svpf_clip_analyse(an.handle, sb.handle, host_frames.ctypes.data, nf, 0, nf,
                                            out_host.ctypes.data)
            if rc:
                raise RuntimeError(sv.lib().svpf_last_error().decode())

        e2e_step()  # the call's own device buffers are allocated on first use
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            e2e_step()
        e2e_value = nf * world * args.e2e_steps / _max_over_ranks(torch, dist, world, time.perf_counter() - t0, dev)
        same = bool(np.array_equal(out_host, pay_host))
    line = None
    if rank == 0:
        peak, peak_kind = _peaks()
        alg_analyse = nf * (2 * fb + pl)
        alg_super = nf * (sb.source_len() + fb)
        roof = {
            "kernel": "analyse_kernel, uint16 build (one CTA per frame pair, fwd/bwd halves)",
            "bound": "hbm", "achieved": alg_analyse / (a_ms / 1000) / 1e9, "peak": peak, "unit": "GB/s",
            "frac": alg_analyse / (a_ms / 1000) / 1e9 / peak, "traffic": None, "peak_source": peak_kind,
            "algorithmic_bytes_per_launch": alg_analyse, "avg_launch_ms": a_ms,
            "super": {"bound": "hbm", "achieved": alg_super / (super_ms / 1000) / 1e9, "peak": peak, "unit": "GB/s",
                      "frac": alg_super / (super_ms / 1000) / 1e9 / peak, "avg_launch_ms": super_ms,
                      "algorithmic_bytes_per_launch": alg_super},
        }
        cpu, parity = None, None
        if not args.no_cpu:
            threads = os.cpu_count() or 1
            pairs = min(args.cpu_pairs or threads, nf - 1)
            so = orc.super_opts(w, h, SUPER_OPT[wl])
            ao = orc.analyse_opts(orc.sdata(so), ANALYSE_OPT[wl], None, w, h)
            orc.total_counters(reset=True, px16=True)
            t0 = time.perf_counter()
            sup_cpu = orc.build_super_many16(so, host_frames[: pairs + 1], threads)
            pay_cpu = orc.analyse_clip16(ao, so, sup_cpu, 0, pairs, threads)
            dt = time.perf_counter() - t0
            cnt = orc.total_counters(reset=True, px16=True)
            cpu = {"value": pairs / dt, "unit": UNIT, "cores": threads, "kind": "port",
                   "sample": f"output frames 0..{pairs - 1} of the same clip (Super + Analyse) on {threads} host "
                             f"threads, the oracle's uint16 build (scalar SAD/SATD)",
                   "cpu_model": _cpu_model()}
            parity = {"pairs_checked": pairs, "bit_exact": bool(np.array_equal(pay_cpu, pay_host[:pairs]))}
            ops_pair = orc.integer_ops(cnt) / pairs
            int_peak = INT32_LANES_PER_SM * _sm_count() * SM_MAX_MHZ * 1e6
            hbm = {k: roof.pop(k) for k in ("bound", "achieved", "peak", "unit", "frac", "peak_source")}
            roof.update({
                "bound": "int32 pipe", "achieved": ops_pair * nf / (a_ms / 1000) / 1e12, "peak": int_peak / 1e12,
                "unit": "Tops/s", "frac": ops_pair * nf / (a_ms / 1000) / int_peak, "ops_per_pair": ops_pair,
                "evaluations_per_pair": cnt[0] / pairs, "samples_compared_per_pair": (cnt[1] + cnt[2]) / pairs,
                "satd_share": (cnt[3] + cnt[4]) / max(cnt[1] + cnt[2], 1),
                "peak_source": f"nominal: {_sm_count()} SMs x {INT32_LANES_PER_SM} int32 lanes (64 ALU + 64 IMAD on "
                               f"the FMA-heavy pipe) x {SM_MAX_MHZ:.0f} MHz; no measured integer peak exists",
                "hbm": hbm})
        line = {
            "metric": "Analyse frame-pairs/s at 2160p 10-bit (bit-exact to the oracle)", "value": value, "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u16", "data": "synthetic",
            "config": {"workload": f"2160p YUV420P10 (uint16) {nf}-frame synthetic clip per GPU, Super "
                                   f"{SUPER_OPT[wl]}, Analyse {ANALYSE_OPT[wl]} (block 8, overlap 4, exhaustive r8 "
                                   f"at level 0, hex2 above, SATD+chroma, fwd+bwd)",
                       "width": w, "height": h, "frames_per_gpu": nf, "pairs_per_step": nf * world,
                       "l2": f"inputs larger than L2 ({nf} super frames = {nf * fb / 1e9:.1f} GB per GPU)",
                       "generator_s": gen_s},
            "clocks": clk.summary(),
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(host_frames.nbytes),
                    "d2h_bytes_per_step": int(nf * pl), "api": "svpf_clip_analyse (host buffers)",
                    "matches_device_path": same},
            "gpu_launches": int(launches), "roofline": roof, "cpu_baseline": cpu, "parity_vs_oracle": parity,
            "super_ms_per_step": super_ms, "analyse_ms_per_step": a_ms,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def _batch_oracle_sample(torch, dev, b, clips, mix) -> dict:
    """Oracle parity of the batch on a sample: for every (resolution, block) shape of the mix, the
    first and last output frame of its first clip (the last frame pairs with itself), checked
    byte for byte against the CPU restatement on all host threads."""
    from oracle import oracle as orc

    seen, checked, equal = set(), [], True
    jobs = []
    for i, ((sb, an, n), (w, h, _, blk, _)) in enumerate(zip(clips, mix)):
        if (w, h, blk) in seen:
            continue
        seen.add((w, h, blk))
        jobs.append((i, w, h, n, blk))
    threads = os.cpu_count() or 1
    for i, w, h, n, blk in jobs:
        sb, an, _ = clips[i]
        fl = sb.source_len()
        frames = torch.as_tensor(_DevBytes(b.frames_device(i), fl * n), device=dev).cpu().numpy().reshape(n, fl)
        pl = an.payload_len()
        pays = torch.as_tensor(_DevBytes(b.payloads_device(i), pl * n), device=dev).cpu().numpy().reshape(n, pl)
        so = orc.super_opts(w, h, SUPER_OPT["1080p"])
        ao = orc.analyse_opts(orc.sdata(so), analyse_opt_for_block(blk), None, w, h)
        need = sorted({0, 1, n - 1})
        supers = orc.build_super_many(so, frames[need], threads)
        sup = dict(zip(need, supers))
        for f in sorted({0, n - 1}):
            want = orc.analyse(ao, so, sup[f], sup[min(f + 1, n - 1)])
            ok = bool(np.array_equal(want, pays[f]))
            equal = equal and ok
            checked.append({"clip": i, "shape": f"{w}x{h}/b{blk}", "frame": f, "bit_exact": ok})
    return {"pairs_checked": len(checked), "bit_exact": equal, "sample": checked}


def run_batched(args, world: int, rank: int, local: int):
    """Config 4: many clips of uneven size in one persistent launch, against per-clip launches."""
    torch, dist = _init_dist(world, local)
    import svpflow_b200 as sv

    dev = torch.device("cuda", local)
    nclips = args.clips or 64
    mix = batched_mix(nclips, max_len=args.max_len or 240)
    mine = [mix[i] for i in clips_of_rank(len(mix), world, rank)]  # clips are sharded whole across ranks
    c2 = CONFIGS["1080p"]
    clips = []
    t0 = time.perf_counter()
    for (w, h, n, blk, seed) in mine:
        sb = sv.Super(w, h, SUPER_OPT["1080p"])
        an = sv.Analyse(sb.sdata, analyse_opt_for_block(blk), w, h)
        frames = make_clip_device(w, h, n, seed=seed, motion=c2["motion"], objects=c2["objects"],
                                  object_motion=c2["object_motion"], device=dev)
        clips.append((sb, an, frames))
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t0
    b = sv.Batch([(sb, an, fr.shape[0]) for sb, an, fr in clips])
    for i, (_, _, fr) in enumerate(clips):
        torch.as_tensor(_DevBytes(b.frames_device(i), fr.numel()), device=dev).copy_(fr.reshape(-1))
    torch.cuda.synchronize()
    host_frames = [fr.cpu().pin_memory() for _, _, fr in clips]  # for the end-to-end run
    clips = [(sb, an, fr.shape[0]) for sb, an, fr in clips]      # the batch holds the device frames now
    torch.cuda.empty_cache()
    if args.shape:  # a fixed launch shape (no autotune trial): "name" or "name:tiles_per_lane"
        name, _, tpl = args.shape.partition(":")
        b.set_shape(sv.Batch.variants().index(name), int(tpl or 8))
        tune = {"trial_pairs_per_s": None, **b.shape(), "chosen_by": f"fixed by --shape {args.shape} (no autotune trial)"}
    elif args.no_autotune:
        tune = {"trial_pairs_per_s": None, **b.shape(), "chosen_by": "default shape (no autotune trial)"}
    else:
        tune = {**b.autotune(), "chosen_by": "svpf_batch_autotune on this batch"}
    stream = torch.cuda.Stream(dev)
    sh = stream.cuda_stream
    pairs = b.pairs
    for _ in range(args.warmup):
        b.launch(sh)
    b.status(sh)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sv.reset_kernel_launches()
    with ClockSampler(_gpu_id(torch, local)) as clk:
        start.record(stream)
        for _ in range(args.steps):
            b.launch(sh)
        stop.record(stream)
        torch.cuda.synchronize()
    launches = sv.kernel_launches()
    b.status(sh)
    ms = _max_over_ranks(torch, dist, world, start.elapsed_time(stop), dev)
    total_pairs = sum(n for (_, _, n, _, _) in mix)  # all ranks' clips; time is the slowest rank's
    assert world > 1 or total_pairs == pairs
    value = total_pairs * args.steps / (ms / 1000.0)

    # the same clips through the per-clip (plain) path, one launch sequence per clip
    max_sup = max(sb.output_len() * n for sb, _, n in clips)
    max_pay = max(an.payload_len() * n for _, an, n in clips)
    max_scr = max(an.scratch_bytes(n) for _, an, n in clips)
    sup_d = torch.empty(max_sup, dtype=torch.uint8, device=dev)
    pay_d = torch.empty(max_pay, dtype=torch.uint8, device=dev)
    scr_d = torch.empty(max_scr, dtype=torch.uint8, device=dev)
    same = True
    plain_ms = 0.0
    with torch.cuda.stream(stream):
        for i, (sb, an, n) in enumerate(clips):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            sb.build_device(b.frames_device(i), sup_d.data_ptr(), n, sh)
            an.analyse_clip_device(sup_d.data_ptr(), n, 0, n, pay_d.data_ptr(), scr_d.data_ptr(), sh)
            e1.record(stream)
            sv.Analyser.device_status(scr_d.data_ptr(), sh)
            plain_ms += e0.elapsed_time(e1)
            L = an.payload_len() * n
            got = torch.as_tensor(_DevBytes(b.payloads_device(i), L), device=dev)
            same = same and bool(torch.equal(got, pay_d[:L]))
    plain_ms = _max_over_ranks(torch, dist, world, plain_ms, dev)
    plain_value = total_pairs / (plain_ms / 1000.0)
    oracle_check = None
    if rank == 0 and not args.no_cpu:
        oracle_check = _batch_oracle_sample(torch, dev, b, clips, [m for i, m in enumerate(mix) if i % world == rank])

    # end to end through the host-buffer batch call (pinned frames in, payloads out)
    del sup_d, pay_d, scr_d
    host_pay = [torch.empty((n, an.payload_len()), dtype=torch.uint8).pin_memory() for _, an, n in clips]
    hf = [t.numpy() for t in host_frames]
    hp = [t.numpy() for t in host_pay]
    b.run(hf, hp)
    e2e_value = None
    if args.e2e_steps > 0:
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            b.run(hf, hp)
        e2e_s = _max_over_ranks(torch, dist, world, time.perf_counter() - t0, dev)
        e2e_value = total_pairs * args.e2e_steps / e2e_s
    e2e_same = all(bool(np.array_equal(hp[i].reshape(-1), torch.as_tensor(
        _DevBytes(b.payloads_device(i), hp[i].size), device=dev).cpu().numpy())) for i in range(len(clips)))
    if rank == 0:
        res = {}
        for (w, h, n, blk, _) in mix:
            k = f"{w}x{h}/b{blk}"
            res[k] = res.get(k, 0) + n
        line = {
            "metric": "Analyse frame-pairs/s, batched (64 mixed clips, one persistent launch; bit-exact MVs)",
            "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "u8", "data": "synthetic",
            "config": {"workload": f"batched: {nclips} clips, resolution from 640x360/1280x720/1920x1080/2560x1440, "
                                   f"{min(n for _, _, n, _, _ in mix)}-{max(n for _, _, n, _, _ in mix)} frames "
                                   f"(log-uniform 16-{args.max_len or 240}), block 8 or 16 with overlap half a block, "
                                   f"Super {{pel:2}}, UMH r16, SATD + chroma, fwd+bwd",
                       "clips": nclips, "pairs": total_pairs, "pairs_by_shape": res,
                       "l2": "inputs larger than L2", "parallelism": f"clips sharded over {world} GPU(s)",
                       "device_bytes_per_gpu": b.device_bytes, "generation_s": gen_s},
            "launch_shape": tune,
            "clocks": clk.summary(),
            "plain_per_clip": {"value": plain_value, "unit": UNIT, "ms": plain_ms,
                               "how": "Super + svpf_clip_analyse_device per clip, clips one after another"},
            "batched_over_plain": value / plain_value,
            "payloads_equal_plain": same,
            "parity_vs_oracle": oracle_check,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(sum(t.numel() for t in host_frames)),
                    "d2h_bytes_per_step": int(sum(t.numel() for t in host_pay)),
                    "api": "svpf_batch_run (host buffers)", "matches_device_path": e2e_same},
            "gpu_launches": int(launches),
        }
        print(json.dumps(line), flush=True)
    b.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def _served_oracle_sample(clip_desc, frames: np.ndarray, pay: np.ndarray) -> dict:
    """Oracle parity of one served clip: its first and last output frame (the last pairs with
    itself) against the CPU restatement."""
    from oracle import oracle as orc

    _, w, h, n, _ = clip_desc
    so = orc.super_opts(w, h, SUPER_OPT["1080p"])
    ao = orc.analyse_opts(orc.sdata(so), ANALYSE_OPT["1080p"], None, w, h)
    need = sorted({0, 1, n - 1})
    sup = dict(zip(need, orc.build_super_many(so, frames[need], os.cpu_count() or 1)))
    out = []
    for f in sorted({0, n - 1}):
        want = orc.analyse(ao, so, sup[f], sup[min(f + 1, n - 1)])
        out.append({"frame": f, "bit_exact": bool(np.array_equal(want, pay[f]))})
    return {"clip": f"{w}x{h}, {n} frames", "pairs_checked": len(out), "bit_exact": all(o["bit_exact"] for o in out),
            "sample": out}


def run_served(args, world: int, rank: int, local: int):
    """Config 5: Poisson arrivals into the continuous-batching server; per-pair latency."""
    torch, dist = _init_dist(world, local)
    import svpflow_b200 as sv

    dev = torch.device("cuda", local)
    nclips = args.clips or 16
    rates = [float(r) for r in args.rates.split(",") if r]
    c2 = CONFIGS["1080p"]
    base = served_stream(nclips, 1.0, seed=5 + rank, max_len=args.max_len or 600)  # clip shapes (same for every rate)
    handles, frames = {}, []
    t0 = time.perf_counter()
    for (_, w, h, n, seed) in base:
        if (w, h) not in handles:
            sb = sv.Super(w, h, SUPER_OPT["1080p"])
            handles[(w, h)] = (sb, sv.Analyse(sb.sdata, ANALYSE_OPT["1080p"], w, h))
        fr = make_clip_device(w, h, n, seed=seed, motion=c2["motion"], objects=c2["objects"],
                              object_motion=c2["object_motion"], device=dev)
        frames.append(fr.cpu().pin_memory().numpy())
        del fr
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t0
    budget = int(args.budget_gb * (1 << 30))
    total_pairs = sum(n for (_, _, _, n, _) in base)
    # identity: a small clip served alone equals the plain path
    k_small = min(range(nclips), key=lambda i: base[i][3] * base[i][1] * base[i][2])
    sb0, an0 = handles[(base[k_small][1], base[k_small][2])]
    want_small = an0.analyse_clip(sb0, frames[k_small])
    sweep = []
    oracle_small = None
    for wi, rate in enumerate(rates):
        arrivals = [t for (t, _, _, _, _) in served_stream(nclips, rate, seed=5 + rank, max_len=args.max_len or 600)]
        srv = sv.Server(budget, max_active=args.max_active, chunk_pairs=args.chunk)
        ids = []
        if wi == 0:  # warm-up request (not measured)
            rid = srv.submit(sb0, an0, frames[k_small])
            srv.wait(rid)
        if world > 1:
            dist.barrier()
        t_start = srv.now_ns()
        for k, (_, w, h, n, _) in enumerate(base):
            due = t_start + int(arrivals[k] * 1e9)
            while srv.now_ns() < due:
                time.sleep(min(0.002, max(0.0, (due - srv.now_ns()) / 1e9)))
            sb, an = handles[(w, h)]
            ids.append(srv.submit(sb, an, frames[k]))
        lat = []
        done_last = 0
        identical = True
        for k, rid in enumerate(ids):
            pay, done, (arr, adm, fin) = srv.wait(rid)
            lat.extend(((done - arr) / 1e6).tolist())
            done_last = max(done_last, fin)
            if k == k_small:
                identical = bool(np.array_equal(pay, want_small))
                if oracle_small is None and not args.no_cpu:
                    oracle_small = _served_oracle_sample(base[k_small], frames[k_small], pay)
        span_s = (done_last - t_start) / 1e9
        st = srv.stats()
        srv.close()
        lat = np.asarray(lat)
        sweep.append({"rate_clips_per_s": rate, "pairs": total_pairs, "span_s": span_s,
                      "pairs_per_s": total_pairs / span_s, "p50_ms": float(np.percentile(lat, 50)),
                      "p99_ms": float(np.percentile(lat, 99)), "max_ms": float(lat.max()),
                      "peak_active_clips": st["peak_active"], "peak_device_gb": st["peak_device_bytes"] / 2 ** 30,
                      "kernel_launches": st["kernel_launches"], "small_clip_identical_to_alone": identical})
    # the same clips through the plain per-clip host-buffer path (svpf_clip_analyse), one after another
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k, (_, w, h, n, _) in enumerate(base):
        sb, an = handles[(w, h)]
        an.analyse_clip(sb, frames[k])
    plain_s = _max_over_ranks(torch, dist, world, time.perf_counter() - t0, dev)
    plain = {"value": total_pairs / plain_s, "unit": UNIT, "s": plain_s,
             "how": "svpf_clip_analyse (host frames in, payloads out) per clip, clips one after another"}
    for r in sweep:
        r["over_plain"] = r["pairs_per_s"] / plain["value"]
    if rank == 0:
        best = max(sweep, key=lambda r: r["pairs_per_s"])
        line = {
            "metric": "served Analyse frame-pairs/s and p50/p99 per-frame-pair latency (bit-exact MVs)",
            "value": best["pairs_per_s"], "unit": UNIT, "n_gpus": world, "steps": len(rates), "warmup": 1,
            "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u8", "data": "synthetic",
            "config": {"workload": f"served: {nclips} clips per rate, Poisson arrivals, resolution from "
                                   f"360p/720p/1080p/1440p/2160p, 8-{args.max_len or 600} frames log-uniform, "
                                   f"1080p Analyse options, HBM budget {args.budget_gb} GB, {args.max_active} active "
                                   f"clips, chunks of {args.chunk} pairs", "pairs_per_rate": total_pairs,
                       "generation_s": gen_s,
                       "latency": "clip arrival to that pair's payload in host memory"},
            "sweep": sweep,
            "plain_per_clip": plain,
            "parity_vs_oracle": oracle_small,
            "e2e": {"value": best["pairs_per_s"], "unit": UNIT,
                    "h2d_bytes_per_step": int(sum(f.nbytes for f in frames)),
                    "d2h_bytes_per_step": int(sum(handles[(w, h)][1].payload_len() * n for (_, w, h, n, _) in base)),
                    "api": "svpf_server_submit / svpf_server_wait (host buffers)"},
            "gpu_launches": int(sum(r["kernel_launches"] for r in sweep)),
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="svpflow_b200")
    ap.add_argument("--frames", type=int, default=0, help="frames per clip (default: the workload's)")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--cpu-pairs", type=int, default=0, help="CPU baseline sample (0 = one per host thread)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--workload", default="1080p",
                    choices=["1080p", "640x360", "2160p10", "batched", "served", "render"])
    ap.add_argument("--clips", type=int, default=0, help="batched: clips (default 64); served: clips per rate (16)")
    ap.add_argument("--max-len", type=int, default=0, help="longest clip in frames (default: the workload's)")
    ap.add_argument("--rates", default="5,50,200", help="served: arrival rates, clips/s")
    ap.add_argument("--budget-gb", type=float, default=150.0, help="served: HBM budget")
    ap.add_argument("--max-active", type=int, default=8, help="served: clips in flight")
    ap.add_argument("--chunk", type=int, default=32, help="served: output frames per launch")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--shape", default="", help="batched: fixed launch shape name[:tiles_per_lane], no autotune")
    ap.add_argument("--no-lookahead", action="store_true", help="Analyse without look-ahead (A/B timing)")
    ap.add_argument("--size", default="", help="WxH: the 1080p / 640x360 workload's options at another frame size")
    ap.add_argument("--lookahead", type=int, default=5,
                    help="look-ahead bits: 1 level 0, 2 coarser levels, 4 level 0 in its own launch (default 5)")
    ap.add_argument("--shard", default="clips", choices=["clips", "frames"],
                    help="N>1: a clip per GPU (weak scaling, default) or one clip split in frame ranges (strong)")
    ap.add_argument("--no-sub", action="store_true",
                    help="1080p: leave out the batched and served objects of the default line")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank)
    if args.workload == "batched":
        return run_batched(args, world, rank, local)
    if args.workload == "served":
        return run_served(args, world, rank, local)
    if args.workload == "2160p10":
        return run_2160p10(args, world, rank, local)
    if args.workload == "render":
        return run_render(args, world, rank, local)
    global WORKLOAD, METRIC
    if args.workload == "640x360":
        WORKLOAD, METRIC = "640x360", "Analyse frame-pairs/s at 640x360 (bit-exact MVs)"

    import torch
    import torch.distributed as dist

    import svpflow_b200 as sv

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    dev = torch.device("cuda", local)
    c = CONFIGS[WORKLOAD]
    w, h, nf = c["width"], c["height"], args.frames or c["frames"]
    if args.size:  # the workload's options and motion at another frame size (profiling cases; no CPU leg)
        w, h = (int(v) for v in args.size.lower().split("x"))
        args.no_cpu = True
    sb = sv.Super(w, h, SUPER_OPT[WORKLOAD])
    an = sv.Analyse(sb.sdata, ANALYSE_OPT[WORKLOAD], w, h)
    an.set_lookahead(0 if args.no_lookahead else args.lookahead)
    shard_frames = args.shard == "frames" and world > 1
    if shard_frames:  # one clip split into frame ranges (strong scaling): this rank's slice and outputs
        clip = make_clip(w, h, nf, seed=1000, motion=c["motion"], objects=c["objects"],
                         object_motion=c["object_motion"])
        lo, hi, a_first, a_count = shard_clip(nf, an.delta, world, rank)
        clip = np.ascontiguousarray(clip[lo:hi])
        a_first -= lo
    else:  # a clip per rank (weak scaling)
        clip = make_clip(w, h, nf, seed=1000 + rank, motion=c["motion"], objects=c["objects"],
                         object_motion=c["object_motion"])
        a_first, a_count = 0, nf
    n_src = clip.shape[0]  # source frames this rank uploads and builds super frames for
    fb, pl = sb.output_len(), an.payload_len()
    frames_d = torch.from_numpy(clip).to(dev)
    supers_d = torch.empty((n_src, fb), dtype=torch.uint8, device=dev)
    pay_d = torch.empty((a_count, pl), dtype=torch.uint8, device=dev)
    scratch_d = torch.empty(an.scratch_bytes(a_count), dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    sh = stream.cuda_stream

    # inputs smaller than L2: a 256 MB write before every step flushes it (outside the step's events)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev) if WORKLOAD != "1080p" else None

    def step(ev=None):
        if flush is not None:
            flush.fill_(1)
        if ev:
            ev[0].record(stream)
        sb.build_device(frames_d.data_ptr(), supers_d.data_ptr(), n_src, sh)
        if ev:
            ev[1].record(stream)
        an.analyse_clip_device(supers_d.data_ptr(), n_src, a_first, a_count, pay_d.data_ptr(), scratch_d.data_ptr(),
                               sh)
        if ev:
            ev[2].record(stream)

    for _ in range(args.warmup):
        step()
    sv.Analyser.device_status(scratch_d.data_ptr(), sh)
    torch.cuda.synchronize()

    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sv.reset_kernel_launches()
    with ClockSampler(_gpu_id(torch, local)) as clk:
        start.record(stream)
        for i in range(args.steps):
            step(evs[i])
        stop.record(stream)
        torch.cuda.synchronize()
    launches = sv.kernel_launches()
    if world > 1:
        dist.barrier()
    sv.Analyser.device_status(scratch_d.data_ptr(), sh)
    la = sv.Analyser.lookahead_stats(scratch_d.data_ptr(), sh)  # the last step's level-0 look-ahead counters
    ms = start.elapsed_time(stop)
    super_ms = [e[0].elapsed_time(e[1]) for e in evs]
    analyse_ms = [e[1].elapsed_time(e[2]) for e in evs]
    if flush is not None:  # the steps' own time, without the L2 flushes between them
        ms = sum(e[0].elapsed_time(e[2]) for e in evs)
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    total_pairs = nf if shard_frames else nf * world  # output frames of the whole job per step
    value = total_pairs * args.steps / (ms_max / 1000.0)

    # end to end through the host-buffer API: pinned host frames in, payloads out
    pinned = torch.from_numpy(clip).pin_memory()
    host_frames = pinned.numpy()
    out_host = torch.empty((a_count, pl), dtype=torch.uint8).pin_memory().numpy()
    def e2e_step():
        rc = sv.lib().svpf_clip_analyse(an.handle, sb.handle, host_frames.ctypes.data, n_src, a_first, a_count,
                                        out_host.ctypes.data)
        if rc:
            raise RuntimeError(sv.lib().svpf_last_error().decode())

    e2e_value, same = None, None
    if args.e2e_steps > 0:
        e2e_step()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            e2e_step()
        e2e_s = time.perf_counter() - t0
        t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_value = total_pairs * args.e2e_steps / float(t.item())
        same = bool(np.array_equal(out_host, pay_d.cpu().numpy()))

    line = None
    if rank == 0:
        peak, peak_kind = _peaks()
        a_ms = statistics.mean(analyse_ms)
        s_ms = statistics.mean(super_ms)
        alg_analyse = a_count * (2 * fb + pl)  # algorithmic bytes of one Analyse launch: 2 super frames + payload per pair
        alg_super = n_src * (sb.source_len() + fb)  # one Super launch sequence: source read + super frame write
        int_peak = INT32_LANES_PER_SM * _sm_count() * SM_MAX_MHZ * 1e6
        ops_pair = None if args.size else OPS_PER_PAIR.get(WORKLOAD)  # the constants hold at the workload's size
        ops_src = ("no count at this frame size (CPU leg not run)" if args.size else
                   "constant from an earlier oracle count of the same workload (CPU leg not run)")
        cpu = None
        parity = None
        cnt = None
        if not args.no_cpu:
            threads = os.cpu_count() or 1
            pairs = min(args.cpu_pairs or CPU_PAIRS_PER_THREAD * threads, a_count - 1)
            dt, pay_cpu, _ = cpu_reference(nf, threads, pairs, seed=1000 + rank)
            from oracle import oracle as orc

            cnt = cpu_reference.counters
            ops_pair = orc.integer_ops(cnt) / pairs
            ops_src = (f"compares the oracle executed on output frames 0..{pairs - 1} (2 ops per SAD sample, 111 "
                       f"per SATD 4x4 tile)")
        # the Analyse kernel's primary bound: the int32 pipes (no dense contraction, little HBM traffic)
        roof = {
            "kernel": ("Analyse: analyse_kernel (one CTA per frame pair, fwd/bwd halves: the coarser levels), "
                       "analyse_level0_kernel (one CTA per warp: level 0 with look-ahead), analyse_finish_kernel; "
                       "timed together"),
            "bound": "int32 pipe", "unit": "Tops/s", "peak": int_peak / 1e12,
            "achieved": ops_pair * a_count / (a_ms / 1000) / 1e12 if ops_pair else None,
            "frac": ops_pair * a_count / (a_ms / 1000) / int_peak if ops_pair else None,
            "traffic": TRAFFIC_PER_PAIR * a_count if WORKLOAD == "1080p" and not args.size else None,
            "traffic_unit": "bytes per launch",
            "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum of the three kernels of the "
                               "240-pair launch, per pair x pairs"),
            "ops_per_pair": ops_pair, "ops_source": ops_src, "avg_launch_ms": a_ms,
            "peak_source": f"nominal: {_sm_count()} SMs x {INT32_LANES_PER_SM} int32 lanes (64 on the ALU pipe + 64 "
                           f"IMAD on the FMA-heavy pipe) x {SM_MAX_MHZ:.0f} MHz; no measured integer peak exists",
            "decomposition": ROOF_DECOMPOSITION,
            "hbm": {"bound": "hbm", "achieved": alg_analyse / (a_ms / 1000) / 1e9, "peak": peak, "unit": "GB/s",
                    "frac": alg_analyse / (a_ms / 1000) / 1e9 / peak, "peak_source": peak_kind,
                    "algorithmic_bytes_per_launch": alg_analyse,
                    "note": "2 super frames + payload per pair: far from HBM-bound"},
            "super": {"bound": "hbm", "achieved": alg_super / (s_ms / 1000) / 1e9, "peak": peak, "unit": "GB/s",
                      "frac": alg_super / (s_ms / 1000) / 1e9 / peak, "avg_launch_ms": s_ms,
                      "algorithmic_bytes_per_launch": alg_super, "peak_source": peak_kind},
        }
        if cnt is not None:
            roof["evaluations_per_pair"] = cnt[0] / pairs
            roof["samples_compared_per_pair"] = (cnt[1] + cnt[2]) / pairs
            roof["satd_share"] = (cnt[3] + cnt[4]) / max(cnt[1] + cnt[2], 1)
        if not args.no_cpu:
            cpu = {"value": pairs / dt, "unit": UNIT, "cores": threads, "kind": "port",
                   "sample": f"output frames 0..{pairs - 1} of the same clip (Super + Analyse), "
                             f"{pairs / threads:.1f} frame pairs per host thread on {threads} threads (throughput), "
                             f"oracle/ C restatement of the reference (AVX2 interior SAD/SATD)",
                   "cpu_model": _cpu_model(), "one_core": _one_core()}
            parity = {"pairs_checked": pairs,
                      "bit_exact": bool(np.array_equal(pay_cpu, pay_d[:pairs].cpu().numpy()))}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "strong" if shard_frames else "weak",
            "vs_baseline": None, "dtype": "u8", "data": "synthetic", "config": _config(nf, world, shard_frames),
            "clocks": clk.summary(),
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(clip.nbytes),
                    "d2h_bytes_per_step": int(a_count * pl), "api": "svpf_clip_analyse (host buffers)",
                    "matches_device_path": same},
            "gpu_launches": int(launches),
            "roofline": roof,
            "cpu_baseline": cpu,
            "parity_vs_oracle": parity,
            "serial_chain": _chain(an, a_count, a_ms),
            "lookahead": {**la, "mode": 0 if args.no_lookahead else args.lookahead,
                          "rerun_fraction": la["reruns"] / la["blocks"] if la["blocks"] else None,
                          "note": "one block per warp in flight; each block re-checks the neighbour seeds "
                                  "committed after it started and re-runs its refinement when one wins "
                                  "(level-0 counters of the last timed step)"},
            "super_ms_per_step": statistics.mean(super_ms), "analyse_ms_per_step": statistics.mean(analyse_ms),
        }
        if args.size:
            line["config"].update(width=w, height=h, workload=f"{w}x{h}: " + line["config"]["workload"])
        if world == 1 and WORKLOAD == "1080p" and not args.no_sub and not args.size:
            # the metric's other two halves (batched vs plain, served p50/p99), each in its own
            # process after this one's buffers are released
            del frames_d, supers_d, pay_d, scratch_d, pinned, out_host
            torch.cuda.synchronize()
            torch.cuda.empty_cache()
            line["batched"] = _sub_batched(args)
            line["served"] = _sub_served(args)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def _sub_line(extra, timeout_s: int) -> dict:
    """Runs this script on another workload in a child process and returns its JSON line."""
    cmd = [sys.executable, os.path.abspath(__file__), *extra]
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout_s)
    except subprocess.TimeoutExpired:
        return {"error": f"{' '.join(extra)}: no result within {timeout_s} s"}
    for ln in reversed(r.stdout.splitlines()):
        if ln.startswith("{"):
            return json.loads(ln)
    return {"error": f"{' '.join(extra)}: rc {r.returncode}: {r.stderr[-600:]}"}


def _sub_batched(args) -> dict:
    """Config 4 in the default line: the 64-clip mix in one persistent launch (CUDA-graph replay)
    against the same clips through the plain per-clip path, with oracle parity on a sample."""
    extra = ["--workload", "batched", "--steps", "1", "--warmup", "1", "--e2e-steps", "0", "--shape", BATCH_SHAPE]
    if args.no_cpu:
        extra.append("--no-cpu")
    b = _sub_line(extra, 1500)
    if "error" in b:
        return b
    keep = ("metric", "value", "unit", "ms_per_step", "plain_per_clip", "batched_over_plain", "payloads_equal_plain",
            "parity_vs_oracle", "launch_shape", "clocks", "gpu_launches")
    out = {k: b.get(k) for k in keep}
    out["config"] = {k: b["config"].get(k) for k in ("workload", "clips", "pairs", "pairs_by_shape",
                                                      "device_bytes_per_gpu")}
    out["timing"] = "one graph replay of the whole batch timed with CUDA events after one untimed replay"
    return out


def _sub_served(args) -> dict:
    """Config 5 in the default line: Poisson arrivals into the continuous-batching server at one
    rate below the server's capacity and one above it (the configuration's lowest rate)."""
    extra = ["--workload", "served", "--rates", SERVED_RATES]
    if args.no_cpu:
        extra.append("--no-cpu")
    sl = _sub_line(extra, 1500)
    if "error" in sl:
        return sl
    keep = ("metric", "value", "unit", "sweep", "plain_per_clip", "parity_vs_oracle", "gpu_launches")
    out = {k: sl.get(k) for k in keep}
    out["config"] = sl.get("config")
    return out


if __name__ == "__main__":
    main()
