"""GPU parity: the CUDA Super / Analyse path through the C ABI against the oracle.

Bit-exact comparison (integer work: tolerance zero) of super frames and Analyse
payloads on seeded synthetic clips, over the option space the reference exposes:
pel 1/2/4, bilinear / bicubic / no sub-pixel planes, block 4/8/16/32, overlap modes
0-3, search types 0/2/3/4, SAD and SATD, one or both directions, penalties.
"""
import numpy as np
import pytest

from oracle import oracle as orc
from payload import first_difference

pytestmark = pytest.mark.gpu


def _sv():
    import svpflow_b200 as sv

    return sv


def _clip(w, h, n, seed, **kw):
    from svpflow_b200.synth import make_clip

    return make_clip(w, h, n, seed=seed, **kw)


SUPER_CASES = [
    (640, 360, "{pel:1}"),
    (640, 360, "{pel:2}"),
    (640, 360, "{pel:4}"),
    (320, 240, "{pel:2, gpu:0}"),          # bicubic sub-pixel planes
    (320, 240, "{pel:2, gpu:0, scale:{up:0}}"),
    (320, 240, "{pel:2, gpu:2}"),          # no sub-pixel planes
    (320, 240, "{pel:1, full:false}"),
    (192, 108, "{pel:2, scale:{down:2}}"),  # no pyramid reduction
    (66, 38, "{pel:2}"),                    # widths that are not multiples of 4
    (1920, 1080, "{pel:2}"),
]


@pytest.mark.parametrize("w,h,opt", SUPER_CASES)
def test_super_matches_oracle(w, h, opt):
    sv = _sv()
    clip = _clip(w, h, 2, seed=w * 7 + h)
    sb = sv.Super(w, h, opt)
    so = orc.super_opts(w, h, opt)
    assert sb.sdata == orc.sdata(so) and sb.super_height == orc.super_height(so)
    got = sb.build_many(clip)
    for i in range(clip.shape[0]):
        want = orc.build_super(so, clip[i])
        if not np.array_equal(got[i], want):
            bad = np.nonzero(got[i] != want)[0]
            pytest.fail(f"frame {i}: {len(bad)} bytes differ, first at {bad[0]} (row {bad[0] // w})")


MANY_CASES = [  # launches of at least 50 frames take the one-CTA-per-frame-and-plane pyramid kernel
    (192, 108, "{pel:2}", 50),
    (320, 240, "{pel:1, full:false}", 52),  # fewer super-frame rows than the level-0 region
    (640, 360, "{pel:4}", 50),
    (1280, 720, "{pel:2}", 50),
    (200, 120, "{pel:2}", 60),               # widths that are not multiples of 16: the per-row kernels
]


@pytest.mark.parametrize("w,h,opt,n", MANY_CASES)
def test_super_many_frames_matches_oracle(w, h, opt, n):
    import os

    sv = _sv()
    clip = _clip(w, h, n, seed=w + 3 * h)
    sb = sv.Super(w, h, opt)
    so = orc.super_opts(w, h, opt)
    got = sb.build_many(clip)
    want = orc.build_super_many(so, clip, os.cpu_count() or 1)
    for i in range(n):
        if not np.array_equal(got[i], want[i]):
            bad = np.nonzero(got[i] != want[i])[0]
            pytest.fail(f"frame {i}: {len(bad)} bytes differ, first at {bad[0]}")


ANALYSE_CASES = [
    # (w, h, super opt, analyse opt, frames)
    (640, 360, "{pel:1}", "{block:{w:16,overlap:0},main:{search:{type:2,distance:2,satd:false,coarse:{satd:false}}}}", 3),
    (320, 180, "{pel:2}", "{block:{w:16,overlap:3},main:{search:{type:3,distance:16,satd:true}}}", 3),
    (256, 144, "{pel:2}", "{}", 2),                                        # defaults: exhaustive r2, overlap 2
    (256, 144, "{pel:1}", "{block:{w:8,overlap:3},main:{search:{type:4,distance:8,satd:true,coarse:{type:2}}}}", 2),
    (256, 144, "{pel:4}", "{block:{w:8,overlap:3},main:{search:{type:4,distance:4,satd:true,coarse:{type:2}}}}", 2),
    (256, 160, "{pel:2}", "{block:{w:32,overlap:1},main:{search:{type:3,distance:8}}}", 2),
    (192, 128, "{pel:2}", "{block:{w:4,overlap:0},main:{search:{type:2,distance:4}}}", 2),
    (192, 128, "{pel:2}", "{block:{w:8,overlap:2},main:{search:{type:0}}}", 2),
    (192, 128, "{pel:2}", "{vectors:1,block:{w:16,overlap:2},main:{search:{type:3,distance:6}}}", 2),
    (192, 128, "{pel:2}", "{vectors:2,block:{w:16,overlap:2},main:{search:{type:2,distance:6}}}", 2),
    (192, 128, "{pel:1}", "{block:{w:16},main:{search:{distance:0}}}", 2),  # level-0 search off
    (192, 128, "{pel:2}", "{main:{penalty:{pnew:-300,pzero:-50,prev:40},search:{type:2,distance:4}}}", 2),
    (192, 128, "{pel:2}", "{main:{search:{coarse:{distance:-6,bad:{range:5}}}}}", 2),
    (192, 128, "{pel:2}", "{main:{search:{coarse:{bad:{sad:30}}},penalty:{lambda:3,plevel:2}}}", 2),
    (256, 144, "{pel:2}", "{block:{w:16,h:8,overlap:2},main:{search:{type:3,distance:6,satd:true}}}", 2),
    # refine[0].thsad set: exact_recalculate onto half-size output blocks
    (192, 128, "{pel:2}", "{refine:[{thsad:200,search:{type:2,distance:3,satd:true}}]}", 2),
    (256, 144, "{pel:2}", "{block:{w:16,overlap:2},main:{search:{type:3,distance:6}},refine:[{thsad:50}]}", 2),
    (192, 128, "{pel:4}", "{block:{w:8,overlap:0},refine:[{thsad:0,search:{type:4,distance:2}}]}", 2),
    (160, 96, "{pel:1}", "{vectors:1,block:{w:32,overlap:1},refine:[{thsad:100,search:{type:3,distance:8}}]}", 2),
    (192, 128, "{pel:2}", "{vectors:2,main:{penalty:{pnew:90}},refine:[{thsad:20000,search:{type:2}}]}", 2),
]


@pytest.mark.parametrize("case", range(len(ANALYSE_CASES)))
def test_analyse_matches_oracle(case):
    sv = _sv()
    w, h, sopt, aopt, n = ANALYSE_CASES[case]
    clip = _clip(w, h, n, seed=100 + case, motion=6, objects=3, object_motion=10)
    sb = sv.Super(w, h, sopt)
    an = sv.Analyse(sb.sdata, aopt, w, h)
    so = orc.super_opts(w, h, sopt)
    ao = orc.analyse_opts(orc.sdata(so), aopt, None, w, h)
    assert an.vector_header() == orc.vdata_header(ao)
    supers = sb.build_many(clip)
    got = an.analyse_clip(sb, clip)
    for i in range(n):
        j = min(i + max(ao.delta, 1), n - 1)
        want = orc.analyse(ao, so, supers[i], supers[j])
        assert got[i].tobytes() == want.tobytes(), f"output frame {i}: " + first_difference(got[i], want)


def test_analyse_full_1080p_matches_oracle():
    """The benchmark's own configuration at its full frame size: 1920x1080, Super {pel:2}, block 16,
    overlap 8, UMH r16, SATD + chroma, both directions, over 3 frames of the seeded benchmark clip
    (motion ranges of the 1080p workload); output frame 2 is the last frame paired with itself
    (analyse_filter.rs:279)."""
    import os

    from svpflow_b200.synth import ANALYSE_OPT, CONFIGS, SUPER_OPT

    sv = _sv()
    c = CONFIGS["1080p"]
    w, h, n = c["width"], c["height"], 3
    clip = _clip(w, h, n, seed=1000, motion=c["motion"], objects=c["objects"], object_motion=c["object_motion"])
    sb = sv.Super(w, h, SUPER_OPT["1080p"])
    an = sv.Analyse(sb.sdata, ANALYSE_OPT["1080p"], w, h)
    so = orc.super_opts(w, h, SUPER_OPT["1080p"])
    ao = orc.analyse_opts(orc.sdata(so), ANALYSE_OPT["1080p"], None, w, h)
    supers = orc.build_super_many(so, clip, os.cpu_count() or 1)
    assert np.array_equal(sb.build_many(clip), supers)
    want = orc.analyse_clip(ao, so, supers, 0, n, os.cpu_count() or 1)
    got = an.analyse_clip(sb, clip)
    for i in range(n):
        assert got[i].tobytes() == want[i].tobytes(), f"output frame {i}: " + first_difference(got[i], want[i])
