"""Known-answer tests of the oracle's primitives (CPU).

Values are derived by hand from the reference's formulas (crates/svpflow1/src/...) or by an
independent numpy restatement, so a transcription error in oracle/svpf_oracle.c shows up here.
"""
import ctypes
import math

import numpy as np
import pytest

from oracle import oracle as orc
from payload import decode


def test_reduce_dim_and_levels():
    # super_opts.rs:70-87: dim -> 2*(dim/4) per level; levels until a side drops below 4
    assert [orc.reduce_dim(1080, n) for n in range(9)] == [1080, 540, 270, 134, 66, 32, 16, 8, 4]
    assert [orc.reduce_dim(1920, n) for n in range(4)] == [1920, 960, 480, 240]
    assert orc.auto_levels(1920, 1080) == 9
    assert orc.auto_levels(640, 360) == 7
    assert orc.auto_levels(3, 100) == 0


def test_super_height_and_sdata():
    so = orc.super_opts(1920, 1080, "{pel:2}")
    # super_plane_height: pel^2 * h + sum of the coarser levels (super_opts.rs:89-95)
    assert orc.super_height(so) == 4 * 1080 + (540 + 270 + 134 + 66 + 32 + 16 + 8 + 4)
    assert orc.super_height(so) == 5390
    assert so.gpu == 1 and so.scale_up == 0 and so.full == 1 and so.rc == 0
    # pack_data: h | w<<16 | pel<<32 | levels<<40 | gpu<<48 | flags<<56 (super_opts.rs:51-63)
    assert orc.sdata(so) == 1080 | (1920 << 16) | (2 << 32) | (9 << 40) | (1 << 48)
    so1 = orc.super_opts(640, 360, "{pel:1, full:false, rc:true}")
    assert orc.sdata(so1) == 360 | (640 << 16) | (1 << 32) | (7 << 40) | (1 << 48) | (3 << 56)
    assert orc.super_height(so1) == 180 + 90 + 44 + 22 + 10 + 4


@pytest.mark.parametrize("opt,msg", [
    ("{pel:3}", "SVSuper: pel has to be 1 or 2 or 4"),
    ("{gpu:3}", "SVSuper: gpu has to be 0 or 1 or 2"),
    ("{pel:2, full:false}", "SVSuper: can't ignore finest level with high pel value"),
])
def test_super_option_errors(opt, msg):
    with pytest.raises(ValueError, match=msg):
        orc.super_opts(640, 360, opt)


@pytest.mark.parametrize("opt,msg", [
    ("{vectors:0}", "SVAnalyse: vectors must be 1, 2 or 3"),
    ("{block:{w:12}}", "SVAnalyse: block.w must be 4/8/16/32"),
    ("{block:{overlap:4}}", "SVAnalyse: overlap must be 0, 1"),
])
def test_analyse_option_errors(opt, msg):
    so = orc.super_opts(640, 360, "{pel:2}")
    with pytest.raises(ValueError, match=msg):
        orc.analyse_opts(orc.sdata(so), opt)


def test_analyse_levels_grid_lambda():
    so = orc.super_opts(1920, 1080, "{pel:2}")
    ao = orc.analyse_opts(orc.sdata(so), "{block:{w:16,overlap:3},main:{search:{type:3,distance:16,satd:true}}}")
    assert (ao.block_w, ao.block_h, ao.overlap_x, ao.overlap_y) == (16, 16, 8, 8)
    assert ao.levels == 7 == orc.auto_search_levels(1920, 1080, 16, 16, 8, 8)
    assert [orc.level_grid(ao, l) for l in range(7)] == [(239, 134), (120, 67), (60, 33), (30, 16), (15, 8), (7, 4), (3, 2)]
    # lambda = 2*area*1000*0.015625*10 (analyse_opts.rs:176-177); lsad, bad.sad scaled by area/32
    assert ao.lambda_ == 80000 and ao.lsad == 64000 and ao.coarse_bad_sad == 8000
    assert (ao.search_type, ao.coarse_search_type, ao.distance, ao.coarse_distance) == (3, 3, 16, 0)
    assert ao.fine_satd == 1 and ao.coarse_satd == 1 and ao.coarse_bad_range == -24
    assert orc.payload_len(ao) == 0x40 + 2 * (4 + 239 * 134 * 8) == 512488
    # portable Analyser::new keeps the 16x16-scaled lsad of from_opt(None) (portable.rs:203-224)
    ap = orc.analyser_portable(so, 8, 8, 0, 3)
    assert ap.lambda_ == int(64 * 312.5) and ap.lsad == 64000


def _hadamard_np(d):
    h = np.array([[1, 1, 1, 1], [1, -1, 1, -1], [1, 1, -1, -1], [1, -1, -1, 1]])
    return int(np.abs(h @ np.asarray(d).reshape(4, 4) @ h.T).sum())


def test_hadamard4_against_matrix_form():
    rng = np.random.default_rng(3)
    cases = [np.ones(16, int), np.eye(4, dtype=int).ravel(), np.full(16, 255), np.full(16, -255)]
    cases += [rng.integers(-255, 256, 16) for _ in range(200)]
    for d in cases:
        assert orc.hadamard4(d) == _hadamard_np(d)
    assert orc.hadamard4(np.ones(16, int)) == 16


def test_adapt_lambda_formula():
    # adapt_lambda, analyse_search.rs:1555-1564, in f64
    for nl, lsad, score in [(1755, 64000, 1000), (80000, 64000, 0xFFFFFFFF), (3, 1, 0xFFFFFFFF), (0, 1, 0xFFFFFFFF),
                            (100, 64000, 123456), (21474836, 8, 7)]:
        l = float(max(lsad, 1))
        half = -1.0 if score == 0xFFFFFFFF else float(score >> 1)
        try:
            t = l / (l + half)
            v = min(float(nl) * t * t, 21474836.47)
        except ZeroDivisionError:
            v = 21474836.47  # inf or NaN -> f64::min picks 21474836.47
        if math.isnan(v):
            v = 21474836.47
        assert orc.adapt_lambda(nl, lsad, score) == int(v)


def test_rescale_and_global():
    vecs = (orc.Vec8 * 6)()
    data = [(0, 0, 100), (30, 0, 100), (400, 200, 1000), (-5, 3, 50), (2000, 2000, 7), (-5, 4, 0xFFFFFF)]
    for i, (dx, dy, s) in enumerate(data):
        vecs[i].dx, vecs[i].dy, vecs[i].score = dx, dy, s
    gx, gy = ctypes.c_int32(), ctypes.c_int32()
    orc.lib().or_global_doubled(vecs, 6, ctypes.byref(gx), ctypes.byref(gy))
    # mode dx: values -5 (x2) -> mode -5; dy: 0 (x2) -> 0; members within 5: (0,0),(-5,3),(-5,4) -> mean
    sx, sy, n = 0 - 5 - 5, 0 + 3 + 4, 3

    def mean(v):  # (sum + signum(sum) * count / 2) / count with Rust's truncating division
        sgn = (v > 0) - (v < 0)
        return int((v + int(sgn * n / 2)) / n)

    assert (gx.value, gy.value) == (2 * mean(sx), 2 * mean(sy)) == (-6, 4)
    orc.lib().or_rescale_scores(vecs, 6, 1920, 1080, 16)
    diag = int(math.sqrt(1920 ** 2 + 1080 ** 2))
    denom = diag * 16
    for i, (dx, dy, s) in enumerate(data):
        ratio = (100 * (abs(dx) + abs(dy))) // denom
        sc = s
        if ratio >= 51:
            sc = min(sc * 20, 2 ** 31 - 1)
        elif ratio >= 16:
            v71 = ((3926827243 * (s & 0xFFFFFFFF) * (ratio - 15)) & (2 ** 64 - 1)) >> 32
            v71 = v71 - (1 << 32) if v71 >= (1 << 31) else v71
            sc = s + 9 * ((v71 >> 31) + (v71 >> 5))
        assert vecs[i].score == (sc & 0xFFFFFFFF) & 0xFFFFFF


def test_payload_layout_and_vdata():
    from svpflow_b200.synth import make_clip

    w, h = 128, 96
    clip = make_clip(w, h, 2, seed=3)
    so = orc.super_opts(w, h, "{pel:2}")
    ao = orc.analyse_opts(orc.sdata(so), "{block:{w:16,overlap:2},main:{search:{type:2,distance:4}}}")
    s0, s1 = orc.build_super(so, clip[0]), orc.build_super(so, clip[1])
    p = orc.analyse(ao, so, s0, s1)
    d = decode(p)
    hd = d["header"]
    assert hd[:3] == [16, 0xA0, 3] and hd[3:6] == [16, 16, 2] and hd[6] == ao.levels and hd[7] == 0
    assert hd[8:14] == [w, h, 4, 4, (w - 4) // 12, (h - 4) // 12] and hd[14:] == [1, 1]
    assert d["previous"] is not None and d["current"] is not None
    vd = orc.vdata_header(ao)
    assert vd == [0xA0, 3, 16, 16, 2, ao.levels, 0, w, h, 4, 4, hd[12], hd[13], 1, 1, 0]
    # identical frames: every vector is zero and every score is the SAD of a perfect match
    q = decode(orc.analyse(ao, so, s0, s0))
    assert (q["current"]["dx"] == 0).all() and (q["current"]["dy"] == 0).all()
    assert (q["current"]["score"] == 0).all()


def test_super_frame_structure():
    from svpflow_b200.synth import make_clip

    w, h = 64, 48
    f = make_clip(w, h, 1, seed=9)[0]
    so = orc.super_opts(w, h, "{pel:2}")
    sf = orc.build_super(so, f)
    Y = sf[:w * orc.super_height(so)].reshape(-1, w)
    src = f[:w * h].reshape(h, w).astype(int)
    assert (Y[:h] == src).all()                                     # level-0 copy
    hpl = (src[:, :-1] + src[:, 1:] + 1) >> 1                       # bilinear h plane, interior
    assert (Y[h:2 * h, :w - 1] == hpl).all()
    vpl = (src[:-1] + src[1:] + 1) >> 1                              # v plane, rows 1..h-2
    assert (Y[2 * h + 1:3 * h - 1] == vpl[1:]).all()
    assert (Y[2 * h] == src[0]).all()                                # v row 0 is the full row 0
