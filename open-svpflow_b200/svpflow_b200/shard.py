"""Sharding of the Analyse work across processes (one per GPU), no data collective.

Every output frame n of a clip is the pair (n, min(n + delta, nframes - 1))
(crates/svpflow1/src/analyse_filter.rs:277-282) and reads only those two super frames, so
a clip splits into contiguous ranges of output frames; a rank builds super frames for its
range plus a halo of `delta` frames after it. Whole clips are dealt to ranks round-robin in
the batched form."""
from __future__ import annotations


def frame_range(nframes: int, world: int, rank: int) -> tuple:
    """Output frames [first, first + count) of `rank`: contiguous, sizes differing by at most one."""
    base, extra = divmod(nframes, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def halo_range(nframes: int, delta: int, first: int, count: int) -> tuple:
    """Source frames [lo, hi) a rank needs to analyse output frames [first, first + count)."""
    if count <= 0:
        return first, first
    return first, min(first + count - 1 + max(delta, 1), nframes - 1) + 1


def pair_frames(nframes: int, delta: int, n: int) -> tuple:
    """The two frames of output frame n."""
    return n, min(n + max(delta, 1), nframes - 1)


def shard_clip(nframes: int, delta: int, world: int, rank: int) -> tuple:
    """This rank's share of one clip: (lo, hi, first, count) -- source frames [lo, hi) to upload and
    build super frames for, and its output frames [first, first + count) of the clip, which are
    output frames [first - lo, first - lo + count) of the slice [lo, hi) (a slice's last frame pairs
    with itself exactly where the clip's does)."""
    first, count = frame_range(nframes, world, rank)
    lo, hi = halo_range(nframes, delta, first, count)
    return lo, hi, first, count


def analyse_clip_shard(analyser, super_builder, frames, world: int = None, rank: int = None) -> tuple:
    """This process's output frames of one clip (a host array of packed frames) through the GPU path
    (svpf_clip_analyse on its slice): returns (first, payloads) with payloads of output frames
    [first, first + len(payloads)). World and rank default to the initialised process group."""
    import torch.distributed as dist

    if world is None or rank is None:
        inited = dist.is_available() and dist.is_initialized()
        world = dist.get_world_size() if inited else 1
        rank = dist.get_rank() if inited else 0
    lo, hi, first, count = shard_clip(frames.shape[0], analyser.delta, world, rank)
    if count == 0:
        return first, frames[:0]
    return first, analyser.analyse_clip(super_builder, frames[lo:hi], first - lo, count)


def gather_payloads(first: int, payloads, nframes: int, dst: int = 0):
    """Every rank's (first, payloads) joined in frame order on rank `dst` (None elsewhere); host
    objects over the process group (the Analyse path itself exchanges nothing)."""
    import numpy as np
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return payloads
    parts = [None] * dist.get_world_size() if dist.get_rank() == dst else None
    dist.gather_object((first, payloads), parts, dst=dst)
    if dist.get_rank() != dst:
        return None
    parts = sorted((p for p in parts if len(p[1])), key=lambda p: p[0])
    out = np.concatenate([p[1] for p in parts]) if parts else payloads[:0]
    assert out.shape[0] == nframes
    return out


def clips_of_rank(nclips: int, world: int, rank: int) -> list:
    """Whole clips dealt round-robin (the batched form)."""
    return [i for i in range(nclips) if i % world == rank]


def max_over_ranks(value: float, device=None) -> float:
    """The slowest rank's time (a no-op without an initialised process group)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
