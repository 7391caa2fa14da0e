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

from svpflow_b200.synth import ANALYSE_OPT, CONFIGS, SUPER_OPT, make_clip  # noqa: E402

WORKLOAD = "1080p"
METRIC = "Analyse frame-pairs/s at 1080p (bit-exact MVs)"
UNIT = "frame-pairs/s"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _config(nframes: int, world: int) -> dict:
    c = CONFIGS[WORKLOAD]
    return {
        "workload": f"1080p YUV420P8 {nframes}-frame synthetic clip per GPU, Super {SUPER_OPT[WORKLOAD]}, "
                    f"Analyse {ANALYSE_OPT[WORKLOAD]} (block 16, overlap 8, UMH r16, SATD+chroma, fwd+bwd)",
        "width": c["width"], "height": c["height"], "frames_per_gpu": nframes,
        "pairs_per_step": nframes * world,
        "l2": "inputs larger than L2 (240 super frames = 3.7 GB per GPU)",
        "parallelism": f"dp{world} (frame ranges per GPU, no collective)" if world > 1 else "single GPU",
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


def cpu_reference(nframes_total: int, threads: int, pairs: int, seed: int = 1000):
    """Times the oracle (CPU restatement of the reference) on `pairs` output frames of the
    workload: Super over the frames they need, then Analyse, on `threads` host threads."""
    from oracle import oracle as orc

    c = CONFIGS[WORKLOAD]
    w, h = c["width"], c["height"]
    n = pairs + 1
    clip = make_clip(w, h, n, seed=seed, motion=c["motion"], objects=c["objects"], object_motion=c["object_motion"])
    so = orc.super_opts(w, h, SUPER_OPT[WORKLOAD])
    ao = orc.analyse_opts(orc.sdata(so), ANALYSE_OPT[WORKLOAD], None, w, h)
    t0 = time.perf_counter()
    supers = orc.build_super_many(so, clip, threads)
    pay = orc.analyse_clip(ao, so, supers, 0, pairs, threads)
    dt = time.perf_counter() - t0
    return dt, pay, clip


def run_reference(args, rank: int):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    pairs = min(max(args.cpu_pairs or threads, 2), 239)
    times = []
    for i in range(args.warmup + args.steps):
        dt, _, _ = cpu_reference(240, threads, pairs, seed=1000 + i)
        if i >= args.warmup:
            times.append(dt)
    total = sum(times)
    value = pairs * args.steps / total
    sample = (f"{pairs} consecutive output frames (Super + Analyse, 1080p clip) per step on {threads} host threads; "
              f"oracle/ C restatement of the reference (the Rust reference cannot be built here)")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": _config(240, 1),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="svpflow_b200")
    ap.add_argument("--frames", type=int, default=CONFIGS[WORKLOAD]["frames"])
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--cpu-pairs", type=int, default=0, help="CPU baseline sample (0 = one per host thread)")
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank)

    import torch
    import torch.distributed as dist

    import svpflow_b200 as sv

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    dev = torch.device("cuda", local)
    c = CONFIGS[WORKLOAD]
    w, h, nf = c["width"], c["height"], args.frames
    clip = make_clip(w, h, nf, seed=1000 + rank, motion=c["motion"], objects=c["objects"],
                     object_motion=c["object_motion"])
    sb = sv.Super(w, h, SUPER_OPT[WORKLOAD])
    an = sv.Analyse(sb.sdata, ANALYSE_OPT[WORKLOAD], w, h)
    fb, pl = sb.output_len(), an.payload_len()
    frames_d = torch.from_numpy(clip).to(dev)
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
    if world > 1:
        dist.barrier()
    sv.Analyser.device_status(scratch_d.data_ptr(), sh)
    ms = start.elapsed_time(stop)
    super_ms = [e[0].elapsed_time(e[1]) for e in evs]
    analyse_ms = [e[1].elapsed_time(e[2]) for e in evs]
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = nf * world * args.steps / (ms_max / 1000.0)

    # end to end through the host-buffer API: pinned host frames in, payloads out
    pinned = torch.from_numpy(clip).pin_memory()
    host_frames = pinned.numpy()
    out_host = torch.empty((nf, pl), dtype=torch.uint8).pin_memory().numpy()
    def e2e_step():
        rc = sv.lib().svpf_clip_analyse(an.handle, sb.handle, host_frames.ctypes.data, nf, 0, nf,
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
        e2e_value = nf * world * args.e2e_steps / float(t.item())
        same = bool(np.array_equal(out_host, pay_d.cpu().numpy()))

    line = None
    if rank == 0:
        peak, peak_kind = _peaks()
        a_ms = statistics.mean(analyse_ms)
        s_ms = statistics.mean(super_ms)
        alg_analyse = nf * (2 * fb + pl)  # algorithmic bytes of one Analyse launch: 2 super frames + payload per pair
        alg_super = nf * (sb.source_len() + fb)  # one Super launch sequence: source read + super frame write
        roof = {
            "kernel": "analyse_kernel (one CTA per frame pair, fwd/bwd halves)",
            "bound": "hbm", "achieved": alg_analyse / (a_ms / 1000) / 1e9, "peak": peak, "unit": "GB/s",
            "frac": alg_analyse / (a_ms / 1000) / 1e9 / peak, "traffic": None, "peak_source": peak_kind,
            "algorithmic_bytes_per_launch": alg_analyse, "avg_launch_ms": a_ms,
            "note": "integer- and dependency-chain-bound block search; the HBM fraction shows how far from "
                    "HBM-bound it is",
            "super": {"bound": "hbm", "achieved": alg_super / (s_ms / 1000) / 1e9, "peak": peak, "unit": "GB/s",
                      "frac": alg_super / (s_ms / 1000) / 1e9 / peak, "avg_launch_ms": s_ms,
                      "algorithmic_bytes_per_launch": alg_super},
        }
        cpu = None
        parity = None
        if not args.no_cpu:
            threads = os.cpu_count() or 1
            pairs = min(args.cpu_pairs or threads, nf - 1)
            dt, pay_cpu, _ = cpu_reference(nf, threads, pairs, seed=1000 + rank)
            cpu = {"value": pairs / dt, "unit": UNIT, "cores": threads, "kind": "port",
                   "sample": f"output frames 0..{pairs - 1} of the same clip (Super + Analyse) on {threads} host "
                             f"threads, oracle/ C restatement of the reference"}
            parity = {"pairs_checked": pairs,
                      "bit_exact": bool(np.array_equal(pay_cpu, pay_d[:pairs].cpu().numpy()))}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u8", "data": "synthetic", "config": _config(nf, world),
            "clocks": clk.summary(),
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(clip.nbytes),
                    "d2h_bytes_per_step": int(nf * pl), "api": "svpf_clip_analyse (host buffers)",
                    "matches_device_path": same},
            "gpu_launches": int(launches),
            "roofline": roof,
            "cpu_baseline": cpu,
            "parity_vs_oracle": parity,
            "super_ms_per_step": statistics.mean(super_ms), "analyse_ms_per_step": statistics.mean(analyse_ms),
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
