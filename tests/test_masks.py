"""SmoothFps' mask planes (renderer.rs coverage_mask / magnitude_mask / max_mask as svpflow2 core.rs
calls them): the oracle against an independent Python restatement and known answers (CPU), and the
device kernels against the oracle, alone and feeding the masked render (GPU)."""
import math

import numpy as np
import pytest

from oracle import oracle as orc
from payload import decode


def _payloads(w=160, h=96, n=3, sopt="{pel:2}", aopt="{block:{w:16,overlap:2},main:{search:{type:3,distance:8}}}",
              seed=31):
    from svpflow_b200.synth import make_clip

    clip = make_clip(w, h, n, seed=seed, motion=8, objects=2, object_motion=12)
    so = orc.super_opts(w, h, sopt)
    ao = orc.analyse_opts(orc.sdata(so), aopt, None, w, h)
    sup = orc.build_super_many(so, clip)
    return orc.vdata_header(ao), orc.analyse_clip(ao, so, sup, 0, n), (w, h)


def _with_vectors(payload, vd, dx, dy, score, region):
    """The payload with region 0 (previous) or 1 (current) rewritten: u32 dx << 16 | u16 dy, then
    u32 score | luma << 24 per vector."""
    out = payload.copy()
    count = vd[11] * vd[12]
    off = 0x40 + 4 + region * (4 + 8 * count)
    words = np.zeros((count, 2), dtype=np.uint32)
    words[:, 0] = (np.asarray(dx, dtype=np.int64).astype(np.uint32) << 16) | (np.asarray(dy, dtype=np.int64) & 0xFFFF)
    words[:, 1] = (np.asarray(score, dtype=np.uint32) & 0xFFFFFF) | (np.uint32(7) << 24)
    out[off: off + 8 * count] = words.reshape(-1).view(np.uint8)
    return out


def _random_field(rng, payload, vd, spread, big=False):
    count = vd[11] * vd[12]
    p = payload
    for region in range(2):
        dx = rng.integers(-spread, spread + 1, size=count)
        dy = rng.integers(-spread, spread + 1, size=count)
        if big:  # a few vectors at the int16 extremes
            idx = rng.integers(0, count, size=max(count // 8, 1))
            dx[idx] = rng.choice([-32768, 32767, -20000, 15000], size=idx.size)
        p = _with_vectors(p, vd, dx, dy, rng.integers(0, 1 << 24, size=count), region)
    return p


# ---------------------------------------------------------------- Python restatement

def _tdiv(a, b):
    if b == 0:
        return 0
    q = abs(a) // abs(b)
    return q if (a >= 0) == (b > 0) else -q


def _sets(payload):
    d = decode(payload)
    prev, cur = d["previous"], d["current"]
    prev = cur if prev is None else prev
    cur = prev if cur is None else cur
    return prev, cur


def _py_cover(vd, rec, mw, mh, cover, t):
    """splat_coverage + window_3x3 + finish_coverage, written as: each vector's four bilinear corner
    weights land on the motion grid where they fall inside it; a clipped 3x3 box sum; then the byte."""
    bw, bh, base, ox, oy, gw, gh = max(vd[2], 1), max(vd[3], 1), max(vd[4], 1), vd[9], vd[10], vd[11], vd[12]
    xs, ys, denom = bw - ox, bh - oy, base * 256
    pts = np.zeros((mh, mw), dtype=np.int64)
    for y in range(gh):
        for x in range(gw):
            k = y * gw + x
            sx = x * xs + _tdiv(t * int(rec["dx"][k]), denom)
            sy = y * ys + _tdiv(t * int(rec["dy"][k]), denom)
            left, top = sx // xs, sy // ys
            lw, tw = (left + 1) * xs - sx, (top + 1) * ys - sy
            for cx, cy, wgt in ((left, top, lw * tw), (left + 1, top, tw * (bw - lw)),
                                (left + 1, top + 1, (bw - lw) * (bh - tw)), (left, top + 1, lw * (bh - tw))):
                if 0 <= cx < mw and 0 <= cy < mh:
                    pts[cy, cx] += wgt
    pad = np.pad(pts, 1)
    win = sum(pad[j: j + mh, i: i + mw] for j in range(3) for i in range(3))
    area = bw * bh
    out = np.zeros((mh, mw), dtype=np.uint8)
    for (y, x), s in np.ndenumerate(win):
        rem = max(area - (int(s) >> 3), 0)
        v = int(rem * (cover / 100.0) * 256.0 / area)
        out[y, x] = 255 if v >= 255 else v & 0xFF
    return out


def _area_values(vd, rec, mw, mh, scale, sharp):
    """magnitude_mask's value per motion-grid point before the byte clamp (floats)."""
    bw, bh, gw, gh = max(vd[2], 1), max(vd[3], 1), vd[11], vd[12]
    area = bw * bh
    out = np.zeros((mh, mw), dtype=np.float64)
    for y in range(mh):
        for x in range(mw):
            k = y * gw + min(x, gw - 1) if y < gh else (gh - 1) * gw
            out[y, x] = math.pow(4.0 * int(rec["score"][k]) * scale / area, sharp) * 255.0
    return out


def _clamp_u8(v):
    return np.where(~np.isfinite(v) | (v <= 0), 0, np.where(v >= 255, 255, np.trunc(np.nan_to_num(v)))).astype(np.uint8)


def _py_masks(vd, payload, phase, cover, scale, sharp):
    mw, mh = orc.vector_grid(vd)
    prev, cur = _sets(payload)
    a0 = _clamp_u8(_area_values(vd, prev, mw, mh, scale, sharp))
    a1 = _clamp_u8(_area_values(vd, cur, mw, mh, scale, sharp))
    return np.stack([_py_cover(vd, cur, mw, mh, cover, 256 - phase), _py_cover(vd, prev, mw, mh, cover, phase),
                     a0, a1, np.maximum(a0, a1)])


# ---------------------------------------------------------------- CPU

CPU_CASES = [  # analyse opt, phase, cover, area scale, area sharp, random field (0 none, spread), big vectors
    ("{block:{w:16,overlap:2},main:{search:{type:3,distance:8}}}", 128, 100, 1.0, 1.0, 0, False),
    ("{block:{w:16,overlap:2},main:{search:{type:3,distance:8}}}", 0, 100, 0.0256, 1.0, 0, False),
    ("{block:{w:8,overlap:0},main:{search:{type:2,distance:4}}}", 256, 37, 0.01, 0.6, 0, False),
    ("{block:{w:8,overlap:3},main:{search:{type:2,distance:4}}}", 77, 250, 0.002, 2.5, 300, False),
    ("{block:{w:32,overlap:3}}", 200, 100, 0.0137, 1.0, 900, True),
    ("{block:{w:16,h:8,overlap:3}}", 1, 0, 1.0, 1.0, 64, False),
]


@pytest.mark.parametrize("case", range(len(CPU_CASES)))
def test_oracle_masks_match_python_restatement(case):
    aopt, phase, cover, scale, sharp, spread, big = CPU_CASES[case]
    vd, pays, _ = _payloads(aopt=aopt, n=2, seed=40 + case)
    p = pays[0]
    if spread:
        p = _random_field(np.random.default_rng(case), p, vd, spread, big)
    got = orc.render_masks(vd, p, phase, cover, scale, sharp)
    want = _py_masks(vd, p, phase, cover, scale, sharp)
    names = ("cover0", "cover1", "area0", "area1", "area_max")
    for k in range(5):
        assert np.array_equal(got[k], want[k]), f"{names[k]}: {np.argwhere(got[k] != want[k])[:4]}"


def test_oracle_masks_known_answers():
    # zero vectors, no overlap, a grid that covers the frame exactly: each vector puts its whole
    # area on its own point, so a window holds 9 (interior), 6 (edge) or 4 (corner) areas:
    # covered = 9a/8 >= a -> 0; 6a/8 -> remaining a/4 -> 64; 4a/8 -> a/2 -> 128
    vd, pays, (w, h) = _payloads(w=160, h=96, n=2, aopt="{block:{w:16,overlap:0},main:{search:{type:2,distance:2}}}")
    gw, gh = vd[11], vd[12]
    assert orc.vector_grid(vd) == (gw, gh) == (10, 6)
    area = 16 * 16
    score = np.full(gw * gh, area // 8)  # 4 * (a / 8) / a * 255 = 127.5 -> 127
    p = pays[0]
    for region in range(2):
        p = _with_vectors(p, vd, np.zeros(gw * gh), np.zeros(gw * gh), score, region)
    m = orc.render_masks(vd, p, 100, 100, 1.0, 1.0)
    want = np.zeros((gh, gw), dtype=np.uint8)
    want[0, :] = want[-1, :] = want[:, 0] = want[:, -1] = 64
    want[0, 0] = want[0, -1] = want[-1, 0] = want[-1, -1] = 128
    assert np.array_equal(m[0], want) and np.array_equal(m[1], want)
    assert (m[2:] == 127).all()
    # cover 0 leaves nothing to cover; cover 200 doubles and clamps
    assert (orc.render_masks(vd, p, 100, 0, 1.0, 1.0)[:2] == 0).all()
    assert orc.render_masks(vd, p, 100, 200, 1.0, 1.0)[0][0, 0] == 255


def test_oracle_masks_fill_past_the_grid():
    # magnitude_mask: columns past the vector grid repeat the row's last vector; rows past it repeat
    # the grid's bottom-left vector
    vd, pays, (w, h) = _payloads(w=168, h=100, n=2, aopt="{block:{w:16,overlap:0},main:{search:{type:2,distance:2}}}")
    gw, gh = vd[11], vd[12]
    mw, mh = orc.vector_grid(vd)
    assert (mw, mh) == (gw + 1, gh + 1)
    score = np.arange(gw * gh) * 9
    p = pays[0]
    for region in range(2):
        p = _with_vectors(p, vd, np.zeros(gw * gh), np.zeros(gw * gh), score, region)
    m = orc.render_masks(vd, p, 128, 100, 1.0, 1.0)
    assert np.array_equal(m[2][:gh, gw], m[2][:gh, gw - 1])
    assert (m[2][gh, :] == m[2][gh - 1, 0]).all()


def test_oracle_masks_reject_undecodable():
    vd, pays, _ = _payloads(n=2)
    bad = pays[0].copy()
    bad[8] ^= 3
    assert orc.render_masks(vd, bad, 128) is None


def test_mask_scratch_size_host_side():
    import svpflow_b200 as sv

    vd, _, _ = _payloads(n=2)
    mw, mh = sv.vector_grid(vd)
    assert sv.render_masks_scratch(vd, 3) == 3 * 2 * (mw + 2) * (mh + 2) * 4
    bad = list(vd)
    bad[9] = bad[2]  # overlap == block
    with pytest.raises(ValueError):
        sv.render_masks_scratch(bad, 1)
    with pytest.raises(ValueError):
        sv.render_masks_scratch([0] * 16, 1)


# ---------------------------------------------------------------- GPU

def _device_masks(vd, pays, phase, cover, scale, sharp):
    import torch

    import svpflow_b200 as sv

    n = pays.shape[0]
    mw, mh = sv.vector_grid(vd)
    src = torch.from_numpy(np.ascontiguousarray(pays)).cuda()
    masks = torch.full((n, 5 * mw * mh), 3, dtype=torch.uint8, device="cuda")
    scratch = torch.empty(sv.render_masks_scratch(vd, n), dtype=torch.uint8, device="cuda")
    status = torch.full((n,), 9, dtype=torch.int32, device="cuda")
    sv.render_masks_device(vd, src.data_ptr(), pays.shape[1], n, phase, masks.data_ptr(), scratch.data_ptr(),
                           status.data_ptr(), cover=cover, area_scale=scale, area_sharp=sharp)
    torch.cuda.synchronize()
    return masks.cpu().numpy().reshape(n, 5, mh, mw), status.cpu().numpy()


GPU_CASES = [  # w, h, analyse opt, phases, cover, area scale, area sharp, random spread, big vectors
    (320, 240, "{block:{w:16,overlap:2},main:{search:{type:3,distance:8,satd:true}}}", (0, 77, 128, 256), 100, 1.0,
     1.0, 0, False),
    (320, 240, "{block:{w:8,overlap:3},main:{search:{type:2,distance:4}}}", (1, 200), 37, 0.0256, 1.0, 0, False),
    (640, 360, "{block:{w:16,overlap:0}}", (128,), 250, 0.01, 1.0, 400, False),
    (256, 144, "{block:{w:32,overlap:3}}", (30, 255), 100, 0.0137, 1.0, 900, True),
    (1920, 1080, "{block:{w:16,overlap:3},main:{search:{type:3,distance:16,satd:true}}}", (100,), 100, 0.0207, 1.0,
     120, False),
    (320, 240, "{block:{w:16,h:8,overlap:3}}", (64, 192), 100, 0.005, 0.6, 200, False),
    (320, 240, "{block:{w:8,overlap:2}}", (128,), 100, 0.002, 2.5, 50, False),
]


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(len(GPU_CASES)))
def test_device_masks_match_oracle(case):
    w, h, aopt, phases, cover, scale, sharp, spread, big = GPU_CASES[case]
    vd, pays, _ = _payloads(w=w, h=h, n=3, aopt=aopt, seed=60 + case)
    rng = np.random.default_rng(case)
    if spread:
        pays = np.stack([pays[0], _random_field(rng, pays[1], vd, spread, big), pays[2]])
    bad = pays.copy()
    bad[2, 8] ^= 3  # flags word: this payload must not decode
    for phase in phases:
        got, status = _device_masks(vd, bad, phase, cover, scale, sharp)
        assert list(status) == [0, 0, 1]
        assert (got[2] == 3).all(), "an undecodable payload's planes are left as they were"
        for f in range(2):
            want = orc.render_masks(vd, bad[f], phase, cover, scale, sharp)
            assert np.array_equal(got[f], want), f"payload {f} phase {phase}: planes differ"


def _magnitude_byte(score, scale, sharp, area):
    v = math.pow(4.0 * score * scale / area, sharp) * 255.0
    if not math.isfinite(v) or v <= 0.0:
        return 0
    return 255 if v >= 255.0 else int(v)


def _steps(scale, sharp, area):
    """The smallest 24-bit score reaching each magnitude byte 1..255 (2^24: none)."""
    out = []
    for k in range(1, 256):
        lo, hi = 0, 1 << 24
        while lo < hi:
            mid = (lo + hi) // 2
            if _magnitude_byte(mid, scale, sharp, area) >= k:
                hi = mid
            else:
                lo = mid + 1
        out.append(lo)
    return out


@pytest.mark.parametrize("scale,sharp,area", [(0.01, 0.6, 256), (0.002, 2.5, 64), (0.0256, 1.0, 256),
                                              (1.0, 1.5, 1024), (0.3, 0.25, 64), (0.05, 0.001, 256)])
def test_magnitude_byte_is_a_step_function_of_the_score(scale, sharp, area):
    # the premise of the device's exact magnitude bytes: with libm's pow the byte never decreases as
    # the 24-bit score grows, so counting the step scores at or below a score gives its byte
    import bisect

    steps = _steps(scale, sharp, area)
    assert steps == sorted(steps)
    rng = np.random.default_rng(1)
    sample = set(rng.integers(0, 1 << 24, size=20000).tolist())
    sample |= {t + d for t in steps for d in (-2, -1, 0, 1, 2) if 0 <= t + d < (1 << 24)}
    for sc in sorted(sample):
        assert _magnitude_byte(sc, scale, sharp, area) == bisect.bisect_right(steps, sc), sc


@pytest.mark.gpu
@pytest.mark.parametrize("scale,sharp", [(0.01, 0.6), (0.002, 2.5), (0.0256, 1.0), (1.0, 1.5), (0.3, 0.25)])
def test_device_magnitude_bytes_exact_at_every_step(scale, sharp):
    # scores right at, below and above every step of the byte: the device's step count must give
    # the oracle's (libm pow) byte at each of them
    vd, pays, _ = _payloads(w=320, h=240, n=2, aopt="{block:{w:8,overlap:0},main:{search:{type:2,distance:2}}}")
    count = vd[11] * vd[12]
    area = max(vd[2], 1) * max(vd[3], 1)
    steps = sorted({t + d for t in _steps(scale, sharp, area) for d in (-1, 0, 1) if 0 <= t + d < (1 << 24)})
    scores = np.resize(np.array(steps + [0, (1 << 24) - 1], dtype=np.int64), count)
    p = pays[0]
    for region in range(2):
        p = _with_vectors(p, vd, np.zeros(count), np.zeros(count), np.roll(scores, region), region)
    got, status = _device_masks(vd, p[None, :], 128, 100, scale, sharp)
    want = orc.render_masks(vd, p, 128, 100, scale, sharp)
    assert status[0] == 0
    assert np.array_equal(got[0][2:], want[2:]), f"{np.argwhere(got[0][2:] != want[2:])[:4]}"


@pytest.mark.gpu
@pytest.mark.parametrize("scale,sharp", [(0.01, 0.0005), (0.3, 0.0), (0.01, -0.5), (-1.0, 2.0), (-0.5, 0.5),
                                         (-0.02, 3.0), (float("inf"), 1.0), (0.01, float("nan"))])
def test_device_magnitude_bytes_exact_for_every_setting(scale, sharp):
    # settings outside the step table (sharpness below 1e-3 or not positive, negative or non-finite
    # scale): the host tabulates libm's byte over all 2^24 scores as runs, so the device's bytes
    # equal the oracle's (libm pow) at any score; checked at random scores and at the edges
    vd, pays, _ = _payloads(w=320, h=240, n=2, aopt="{block:{w:8,overlap:0},main:{search:{type:2,distance:2}}}")
    count = vd[11] * vd[12]
    rng = np.random.default_rng(17)
    special = [0, 1, 2, 3, 255, 256, (1 << 24) - 2, (1 << 24) - 1] + [1 << k for k in range(24)]
    scores = np.concatenate([np.array(special, dtype=np.int64),
                             rng.integers(0, 1 << 24, size=count, dtype=np.int64),
                             np.exp(rng.uniform(0, math.log(1 << 24), size=count)).astype(np.int64)])[:count]
    p = pays[0]
    for region in range(2):
        p = _with_vectors(p, vd, np.zeros(count), np.zeros(count), np.roll(scores, 7 * region), region)
    got, status = _device_masks(vd, p[None, :], 128, 100, scale, sharp)
    want = orc.render_masks(vd, p, 128, 100, scale, sharp)
    assert status[0] == 0
    assert np.array_equal(got[0][2:], want[2:]), f"{np.argwhere(got[0][2:] != want[2:])[:4]}"


@pytest.mark.gpu
def test_device_masks_reject_bad_arguments():
    import torch

    import svpflow_b200 as sv

    vd, pays, _ = _payloads(n=2)
    mw, mh = sv.vector_grid(vd)
    src = torch.from_numpy(pays).cuda()
    masks = torch.empty((2, 5 * mw * mh), dtype=torch.uint8, device="cuda")
    scratch = torch.empty(sv.render_masks_scratch(vd, 2), dtype=torch.uint8, device="cuda")
    status = torch.empty(2, dtype=torch.int32, device="cuda")
    args = (src.data_ptr(), pays.shape[1], 2)
    for phase in (-1, 257):
        with pytest.raises(ValueError, match="phase"):
            sv.render_masks_device(vd, *args, phase, masks.data_ptr(), scratch.data_ptr(), status.data_ptr())
    with pytest.raises(ValueError, match="aligned"):
        sv.render_masks_device(vd, src.data_ptr() + 1, pays.shape[1], 2, 128, masks.data_ptr(), scratch.data_ptr(),
                               status.data_ptr())
    with pytest.raises(ValueError, match="aligned"):
        sv.render_masks_device(vd, src.data_ptr(), pays.shape[1] - 2, 2, 128, masks.data_ptr(), scratch.data_ptr(),
                               status.data_ptr())
    with pytest.raises(ValueError, match="aligned"):
        sv.vector_planes_device(vd, src.data_ptr() + 2, pays.shape[1], 2, 160, 96, masks.data_ptr(),
                                status.data_ptr())


@pytest.mark.gpu
def test_masked_render_after_device_chain():
    """Super -> Analyse -> vector planes + mask planes -> algorithm 21 / 22 / 23 render, all on the
    device, against the oracle's chain."""
    import torch

    import svpflow_b200 as sv
    from svpflow_b200.synth import make_clip

    w, h, n = 320, 240, 3
    sopt, aopt = "{pel:2}", "{block:{w:16,overlap:2},main:{search:{type:3,distance:8,satd:true}}}"
    clip = make_clip(w, h, n, seed=23, motion=6, objects=3, object_motion=10)
    sb = sv.Super(w, h, sopt)
    an = sv.Analyse(sb.sdata, aopt, w, h)
    so = orc.super_opts(w, h, sopt)
    ao = orc.analyse_opts(orc.sdata(so), aopt, None, w, h)
    st = torch.cuda.current_stream().cuda_stream
    sup_d = torch.empty((n, sb.output_len()), dtype=torch.uint8, device="cuda")
    pay_d = torch.empty((n, an.payload_len()), dtype=torch.uint8, device="cuda")
    scr_d = torch.empty(an.scratch_bytes(n), dtype=torch.uint8, device="cuda")
    frames_d = torch.from_numpy(clip).cuda()
    sb.build_device(frames_d.data_ptr(), sup_d.data_ptr(), n, st)
    an.analyse_clip_device(sup_d.data_ptr(), n, 0, n, pay_d.data_ptr(), scr_d.data_ptr(), st)
    vd = an.vector_header()
    mw, mh = sv.vector_grid(vd)
    planes = torch.empty((n, 4 * mw * mh), dtype=torch.int16, device="cuda")
    status = torch.zeros(n, dtype=torch.int32, device="cuda")
    sv.vector_planes_device(vd, pay_d.data_ptr(), an.payload_len(), n, w, h, planes.data_ptr(), status.data_ptr())
    phase, cover, scale = 96, 100, 0.0256
    masks = torch.empty((n, 5 * mw * mh), dtype=torch.uint8, device="cuda")
    mscr = torch.empty(sv.render_masks_scratch(vd, n), dtype=torch.uint8, device="cuda")
    mstat = torch.zeros(n, dtype=torch.int32, device="cuda")
    sv.render_masks_device(vd, pay_d.data_ptr(), an.payload_len(), n, phase, masks.data_ptr(), mscr.data_ptr(),
                           mstat.data_ptr(), cover=cover, area_scale=scale)
    torch.cuda.synchronize()
    assert (mstat.cpu().numpy() == 0).all()
    sup_h = orc.build_super_many(so, clip)
    pays = orc.analyse_clip(ao, so, sup_h, 0, n)
    hs = orc.super_height(so)
    # SmoothFps' config: the effective block (block - overlap), origin at half the block
    cfg = {"width": w, "height": h, "block_w": vd[2] - vd[9], "block_h": vd[3] - vd[10], "origin_x": vd[2] // 2,
           "origin_y": vd[3] // 2, "grid_w": mw, "grid_h": mh, "chroma_y_div": 2, "source_step": 2}
    offs = [0, w * hs, w * hs + (w // 2) * (hs // 2)]
    lens = [w * hs, (w // 2) * (hs // 2), (w // 2) * (hs // 2)]
    strides = [w, w // 2, w // 2]
    nm = mw * mh
    tlimit = orc.render_threshold_limit(phase, scale)
    for f in range(n - 1):
        mp = orc.vector_planes(vd, pays[f], w, h)
        om = orc.render_masks(vd, pays[f], phase, cover, scale)
        assert np.array_equal(masks[f].cpu().numpy().reshape(5, mh, mw), om)
        for mode22 in (False, True):
            dsts = [torch.zeros((h // (2 if p else 1), w // (2 if p else 1)), dtype=torch.uint8, device="cuda")
                    for p in range(3)]
            b0, b1 = sup_d[f].data_ptr(), sup_d[f + 1].data_ptr()
            pp, mk = planes[f].data_ptr(), masks[f].data_ptr()
            sv.render_masked_device(cfg, phase, scale, mode22, True, [b0 + o for o in offs], strides, lens,
                                    [b1 + o for o in offs], strides, lens, 1, (pp, pp + 2 * nm),
                                    (pp + 4 * nm, pp + 6 * nm), (mk, mk + nm), mk + 4 * nm,
                                    [d.data_ptr() for d in dsts], strides)
            torch.cuda.synchronize()
            for p in range(3):
                pw, ph = strides[p], h // (2 if p else 1)
                srcs = [sup_h[f][offs[p]: offs[p] + lens[p]], sup_h[f + 1][offs[p]: offs[p] + lens[p]]]
                want = orc.render_dual_plane(cfg, p > 0, True, False, 22 if mode22 else 21, phase, srcs, [pw, pw],
                                             [pw * ph, pw * ph], 1, (mp[0], mp[1]), (mp[2], mp[3]), pw, ph,
                                             (om[0], om[1]), om[4], tlimit)
                assert np.array_equal(dsts[p].cpu().numpy(), want), f"frame {f} mode22 {mode22} plane {p}"
    # algorithm 23 at frame 1 as SmoothFps feeds it: the frame's own two sets, the next payload's
    # previous set (next0) and the previous payload's current set (prev1), all from vector planes
    f = 1
    mp = [orc.vector_planes(vd, pays[k], w, h) for k in range(3)]
    om = orc.render_masks(vd, pays[f], phase, cover, scale)
    dsts = [torch.zeros((h // (2 if p else 1), w // (2 if p else 1)), dtype=torch.uint8, device="cuda") for p in range(3)]
    pl = [planes[k].data_ptr() for k in range(3)]
    sets = [(pl[1], pl[1] + 2 * nm), (pl[1] + 4 * nm, pl[1] + 6 * nm), (pl[2], pl[2] + 2 * nm), (pl[0] + 4 * nm, pl[0] + 6 * nm)]
    mk = masks[f].data_ptr()
    b0, b1 = sup_d[f].data_ptr(), sup_d[f + 1].data_ptr()
    sv.render_mode23_device(cfg, phase, True, [b0 + o for o in offs], strides, lens, [b1 + o for o in offs], strides,
                            lens, 1, sets, (mk, mk + nm), mk + 4 * nm, [d.data_ptr() for d in dsts], strides)
    torch.cuda.synchronize()
    for p in range(3):
        pw, ph = strides[p], h // (2 if p else 1)
        srcs = [sup_h[f][offs[p]: offs[p] + lens[p]], sup_h[f + 1][offs[p]: offs[p] + lens[p]]]
        motions = [(mp[1][0], mp[1][1]), (mp[1][2], mp[1][3]), (mp[2][0], mp[2][1]), (mp[0][2], mp[0][3])]
        want = orc.render_mode23_plane(cfg, p > 0, True, phase, srcs, [pw, pw], [pw * ph, pw * ph], 1, motions,
                                       (om[0], om[1]), om[4], pw, ph)
        assert np.array_equal(dsts[p].cpu().numpy(), want), f"algorithm 23, plane {p}"
