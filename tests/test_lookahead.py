"""Level-0 look-ahead (GPU): each warp of a search direction takes its own level-0 block in the
reference's order, searches it without the neighbour vectors other warps have not committed
yet, and re-checks the reference's selection with them before it commits in order, the warps
either in the pair's CTA or (mode bit 4) as CTAs of their own spread over the SMs. The
payloads must equal the oracle's and those of the same launch without look-ahead, byte for
byte, for every launch shape (one to four warps per direction); the counters show that seeds
were deferred and re-checked. Tolerance: zero (integer work)."""
import os

import numpy as np
import pytest

from oracle import oracle as orc
from payload import first_difference

pytestmark = pytest.mark.gpu

CASES = [
    # (w, h, super opt, analyse opt, frames): the 1080p options on a small frame; small blocks
    # with overlap (many row turns per level); exhaustive, hex2 and one-direction searches;
    # penalties that make neighbour seeds win often; a frame barely larger than three blocks
    (320, 180, "{pel:2}", "{block:{w:16,overlap:3},main:{search:{type:3,distance:16,satd:true}}}", 3),
    (192, 128, "{pel:2}", "{block:{w:8,overlap:2},main:{search:{type:4,distance:3,satd:true}}}", 2),
    (256, 144, "{pel:1}", "{vectors:1,block:{w:8,overlap:1},main:{search:{type:2,distance:4}}}", 2),
    (192, 128, "{pel:4}", "{block:{w:16,overlap:2},main:{penalty:{pnbour:-40,pzero:200,pnew:60},"
                          "search:{type:3,distance:6}}}", 2),
    (192, 128, "{pel:2}", "{main:{penalty:{pnew:-300,pnbour:-20},search:{type:2,distance:4}}}", 2),
    (64, 48, "{pel:2}", "{block:{w:16,overlap:0},main:{search:{type:3,distance:4}}}", 2),
    # coarser levels: the bad-SAD expansion (its running count is read at commit), adaptive radius
    (256, 144, "{pel:2}", "{main:{search:{coarse:{bad:{sad:30,range:-4}}}}}", 2),
    (256, 144, "{pel:2}", "{main:{search:{coarse:{distance:-6,bad:{sad:40,range:5}}}}}", 2),
    (320, 180, "{pel:1}", "{block:{w:8,overlap:2},main:{search:{coarse:{type:4,distance:2,bad:{sad:20}}}}}", 2),
]


def _run(an, sb, clip, levels):
    import torch

    import svpflow_b200 as sv

    an.set_lookahead(levels)
    dev = torch.device("cuda", 0)
    n = clip.shape[0]
    frames = torch.from_numpy(clip).to(dev)
    supers = torch.empty((n, sb.output_len()), dtype=torch.uint8, device=dev)
    pay = torch.empty((n, an.payload_len()), dtype=torch.uint8, device=dev)
    scr = torch.empty(an.scratch_bytes(n), dtype=torch.uint8, device=dev)
    st = torch.cuda.current_stream(dev).cuda_stream
    sb.build_device(frames.data_ptr(), supers.data_ptr(), n, st)
    an.analyse_clip_device(supers.data_ptr(), n, 0, n, pay.data_ptr(), scr.data_ptr(), st)
    sv.Analyser.device_status(scr.data_ptr(), st)
    stats = sv.Analyser.lookahead_stats(scr.data_ptr(), st)
    return pay.cpu().numpy(), stats


@pytest.mark.parametrize("case", range(len(CASES)))
def test_lookahead_is_exact(case):
    import svpflow_b200 as sv
    from svpflow_b200.synth import make_clip

    w, h, sopt, aopt, n = CASES[case]
    clip = make_clip(w, h, n, seed=300 + case, motion=6, objects=3, object_motion=12)
    sb = sv.Super(w, h, sopt)
    an = sv.Analyse(sb.sdata, aopt, w, h)
    so = orc.super_opts(w, h, sopt)
    ao = orc.analyse_opts(orc.sdata(so), aopt, None, w, h)
    want = orc.analyse_clip(ao, so, orc.build_super_many(so, clip, os.cpu_count() or 1), 0, n, os.cpu_count() or 1)
    off, st_off = _run(an, sb, clip, 0)
    for levels in (1, 2, 5, 6):  # level 0 in the pair's CTA; the coarser levels; level 0 spread (+ coarser)
        got, _ = _run(an, sb, clip, levels)
        for i in range(n):
            assert got[i].tobytes() == want[i].tobytes(), (f"look-ahead {levels}, output frame {i}: " +
                                                           first_difference(got[i], want[i]))
    on, st = _run(an, sb, clip, 7)
    for i in range(n):
        assert on[i].tobytes() == want[i].tobytes(), f"look-ahead, output frame {i}: " + first_difference(on[i], want[i])
        assert off[i].tobytes() == want[i].tobytes(), f"serial, output frame {i}: " + first_difference(off[i], want[i])
    vd = an.vector_header()
    dirs = 2 if ao.vectors == 3 else 1
    gw, gh = vd[11], vd[12]
    if gw >= 3 and gh >= 3:  # the look-ahead path runs (grids of at least 3 x 3 blocks at level 0)
        assert st["blocks"] == n * dirs * gw * gh
        assert 0 < st["deferred_blocks"] <= st["blocks"] and st["reruns"] <= st["deferred_blocks"]
    assert st_off["blocks"] == 0


def test_lookahead_every_launch_shape_matches_the_oracle():
    """The batch kernel with every compiled shape: 1, 2 or 4 warps per direction (one to four
    blocks in flight), 2 to 8 CTAs per SM."""
    import svpflow_b200 as sv
    from svpflow_b200.synth import make_clip

    mix = [CASES[0], CASES[1], CASES[3]]
    clips, want = [], []
    for k, (w, h, sopt, aopt, n) in enumerate(mix):
        clip = make_clip(w, h, n, seed=400 + k, motion=6, objects=3, object_motion=12)
        sb = sv.Super(w, h, sopt)
        an = sv.Analyse(sb.sdata, aopt, w, h)
        so = orc.super_opts(w, h, sopt)
        ao = orc.analyse_opts(orc.sdata(so), aopt, None, w, h)
        want.append(orc.analyse_clip(ao, so, orc.build_super_many(so, clip, os.cpu_count() or 1), 0, n,
                                     os.cpu_count() or 1))
        clips.append((sb, an, clip))
    b = sv.Batch([(sb, an, clip.shape[0]) for sb, an, clip in clips])
    try:
        for v in range(len(sv.Batch.variants())):
            b.set_shape(v, 8)
            got = b.run([c[2] for c in clips])
            for i, (g, w_) in enumerate(zip(got, want)):
                assert np.array_equal(g, w_), f"shape {sv.Batch.variants()[v]}: clip {i} differs from the oracle"
    finally:
        b.close()


def test_spread_level0_in_several_launches():
    """More pairs than one cooperative level-0 launch holds (296 bidirectional pairs on 148
    SMs): the pairs go in groups, each group's warps in a launch of their own. The 10-bit build
    takes the look-ahead shape at any pair count, so a 700-pair clip runs three groups."""
    import torch

    import svpflow_b200 as sv
    from test_px16 import clip10

    w, h, sopt, aopt, _ = CASES[5]
    n = 700
    clip = clip10(w, h, n, seed=777, motion=3, objects=2, object_motion=6)
    sb = sv.Super(w, h, sopt, bits=10)
    an = sv.Analyse(sb.sdata, aopt, w, h, bits=10)
    so = orc.super_opts(w, h, sopt)
    ao = orc.analyse_opts(orc.sdata(so), aopt, None, w, h)
    want = orc.analyse_clip16(ao, so, orc.build_super_many16(so, clip), 0, n)
    dev = torch.device("cuda", 0)
    st = torch.cuda.current_stream(dev).cuda_stream
    frames = torch.from_numpy(clip.view(np.uint8).copy()).to(dev)
    supers = torch.empty((n, sb.output_len()), dtype=torch.uint8, device=dev)
    pay = torch.empty((n, an.payload_len()), dtype=torch.uint8, device=dev)
    scr = torch.empty(an.scratch_bytes(n), dtype=torch.uint8, device=dev)
    sb.build_device(frames.data_ptr(), supers.data_ptr(), n, st)
    an.set_lookahead(5)
    an.analyse_clip_device(supers.data_ptr(), n, 0, n, pay.data_ptr(), scr.data_ptr(), st)
    sv.Analyser.device_status(scr.data_ptr(), st)
    stats = sv.Analyser.lookahead_stats(scr.data_ptr(), st)
    got = pay.cpu().numpy()
    for i in range(n):
        assert got[i].tobytes() == want[i].tobytes(), f"output frame {i}: " + first_difference(got[i], want[i])
    vd = an.vector_header()
    assert stats["blocks"] == n * 2 * vd[11] * vd[12]


def test_spread_level0_in_a_cuda_graph():
    """The three launches of a spread Analyse (pair kernel, cooperative level-0 kernel, finish
    kernel) captured into a CUDA graph and replayed give the payloads of a direct call."""
    import torch

    import svpflow_b200 as sv
    from svpflow_b200.synth import make_clip

    w, h, sopt, aopt, n = CASES[0]
    clip = make_clip(w, h, n, seed=901, motion=6, objects=3, object_motion=12)
    sb = sv.Super(w, h, sopt)
    an = sv.Analyse(sb.sdata, aopt, w, h)
    an.set_lookahead(5)
    dev = torch.device("cuda", 0)
    frames = torch.from_numpy(clip).to(dev)
    supers = torch.empty((n, sb.output_len()), dtype=torch.uint8, device=dev)
    direct = torch.empty((n, an.payload_len()), dtype=torch.uint8, device=dev)
    replayed = torch.zeros_like(direct)
    scr = torch.empty(an.scratch_bytes(n), dtype=torch.uint8, device=dev)
    st = torch.cuda.current_stream(dev).cuda_stream
    sb.build_device(frames.data_ptr(), supers.data_ptr(), n, st)
    an.analyse_clip_device(supers.data_ptr(), n, 0, n, direct.data_ptr(), scr.data_ptr(), st)
    sv.Analyser.device_status(scr.data_ptr(), st)
    g = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream(dev)
    side.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(side):
        with torch.cuda.graph(g, stream=side):
            an.analyse_clip_device(supers.data_ptr(), n, 0, n, replayed.data_ptr(), scr.data_ptr(),
                                   side.cuda_stream)
    torch.cuda.current_stream(dev).wait_stream(side)
    for _ in range(2):
        g.replay()
    torch.cuda.synchronize()
    sv.Analyser.device_status(scr.data_ptr(), st)
    assert torch.equal(direct, replayed)
    del g
