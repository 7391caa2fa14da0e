"""The multi-process path on CPU (gloo, world size 2): frame ranges with their halos cover a
clip exactly once; the library's analyse_clip_shard / gather_payloads, with each rank analysing
only its own slice of source frames, reproduce the single-process payloads; the timing
reduction takes the slowest rank. The CUDA library cannot run here, so the analyser these
ranks call is a stand-in with the library's analyse_clip signature that computes with the
oracle (the checker); the sharding code under test is the product's."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from svpflow_b200.shard import (analyse_clip_shard, clips_of_rank, frame_range, gather_payloads, halo_range,
                                max_over_ranks, pair_frames, shard_clip)

W, H, N, SOPT, AOPT = 96, 64, 7, "{pel:2}", "{delta:2,block:{w:8,overlap:2},main:{search:{type:2,distance:3}}}"


def test_ranges_cover_every_output_frame_once():
    for n in (1, 2, 7, 240):
        for world in (1, 2, 3, 8):
            got = []
            for r in range(world):
                first, count = frame_range(n, world, r)
                got += list(range(first, first + count))
                lo, hi = halo_range(n, 2, first, count)
                for k in range(first, first + count):
                    a, b = pair_frames(n, 2, k)
                    assert lo <= a < hi and lo <= b < hi
            assert got == list(range(n))
    assert sorted(sum((clips_of_rank(10, 3, r) for r in range(3)), [])) == list(range(10))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [os.path.join(root, "open-svpflow_b200"), root]
    from oracle import oracle as orc
    from svpflow_b200.synth import make_clip

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        clip = make_clip(W, H, N, seed=21)
        so = orc.super_opts(W, H, SOPT)
        ao = orc.analyse_opts(orc.sdata(so), AOPT, None, W, H)
        seen = []

        class _OracleAnalyser:  # the library's Analyser.analyse_clip signature, computed by the oracle
            delta = ao.delta

            def analyse_clip(self, _sb, frames, first, count):
                seen.append(frames.shape[0])  # only this rank's slice of source frames arrives here
                return orc.analyse_clip(ao, so, orc.build_super_many(so, frames), first, count)

        first, pays = analyse_clip_shard(_OracleAnalyser(), None, clip)
        lo, hi, f2, count = shard_clip(N, ao.delta, world, rank)
        assert first == f2 and len(pays) == count and seen == [hi - lo]
        joined = gather_payloads(first, pays, N)
        slowest = max_over_ranks(1.0 + rank)
        if rank == 0:
            full = orc.analyse_clip(ao, so, orc.build_super_many(so, clip), 0, N)
            out.put((bool(np.array_equal(joined, full)), slowest))
        else:
            assert joined is None
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reproduce_the_single_process_payloads():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        same, slowest = q.get(timeout=300)
    finally:
        for p in procs:
            p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    assert same and slowest == 2.0
