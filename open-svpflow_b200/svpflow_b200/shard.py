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
