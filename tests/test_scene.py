"""SmoothFps's scene class of a payload (metadata.rs analyze_scene = luma_map + classify_scene, as
svpflow2 core.rs scene_class calls it): the oracle against an independent Python restatement (CPU),
and the device kernel against the oracle (GPU, exact), on real payloads and on payloads whose scores
and luma bytes are set to reach every class, every threshold and the luma byte's wrap-around."""
import math

import numpy as np
import pytest

from oracle import oracle as orc
from payload import decode


def _payloads(w=192, h=128, n=3, aopt="{block:{w:16,overlap:2},main:{search:{type:3,distance:8}}}", seed=51):
    from svpflow_b200.synth import make_clip

    clip = make_clip(w, h, n, seed=seed, motion=8, objects=3, object_motion=12)
    so = orc.super_opts(w, h, "{pel:2}")
    ao = orc.analyse_opts(orc.sdata(so), aopt, None, w, h)
    sup = orc.build_super_many(so, clip)
    return orc.vdata_header(ao), orc.analyse_clip(ao, so, sup, 0, n)


def _with_scores(payload, vd, region, score, luma):
    """Region 0 (previous) or 1 (current) with its score and luma words rewritten."""
    out = payload.copy()
    count = vd[11] * vd[12]
    off = 0x40 + 4 + region * (4 + 8 * count)
    words = out[off: off + 8 * count].view(np.uint32).reshape(count, 2).copy()
    words[:, 1] = (np.asarray(score, dtype=np.uint32) & 0xFFFFFF) | (np.asarray(luma, dtype=np.uint32) << 24)
    out[off: off + 8 * count] = words.reshape(-1).view(np.uint8)
    return out


def _py_scene(vd, payload, gamma=1.5, blocks=20, zero=200, m1=1600, m2=2800, scene=4000):
    d = decode(payload)
    prev, cur = d["previous"], d["current"]
    if prev is None and cur is None:
        return 3
    prev = cur if prev is None else prev
    cur = prev if cur is None else cur
    denom = 510.0 if vd[4] == 3 else 255.0
    counts = [0, 0, 0, 0]  # considered, scene, m2, m1
    for i in range(vd[11] * vd[12]):
        value = (float(prev["luma"][i]) + float(cur["luma"][i])) / denom
        byte = max(int(math.pow(value, gamma) * 255.0), 20) & 0xFF
        luma = max(byte, 1)
        score = min(int(cur["score"][i]) * 255, 2**31 - 1) // luma
        if score < zero:
            continue
        counts[0] += 1
        if score >= scene:
            counts[1] += 1
        elif score >= m2:
            counts[2] += 1
        elif score >= m1:
            counts[3] += 1
    required = counts[0] * blocks // 100
    high = counts[1] + counts[2]
    if counts[1] >= required:
        return 3
    if high >= required:
        return 2
    return int(high + counts[3] >= required)


def _cases():
    """(name, vdata, payload, kwargs): real payloads, forced classes, luma wrap, one-set payloads."""
    vd, pays = _payloads()
    out = [("real", vd, p, {}) for p in pays[:2]]
    count = vd[11] * vd[12]
    rng = np.random.default_rng(7)
    # (a frame whose scores all fall below `zero` considers nothing, and 0 >= 0 required makes it a
    # scene change: class 3, as in the reference)
    for target, lo, hi in ((3, 4000, 9000), (2, 2800, 3999), (1, 1600, 2799), (0, 200, 1599), (3, 0, 199)):
        # luma bytes 255 + 255 -> value 2 -> byte (2^1.5 * 255 = 721) & 0xFF = 209; score * 255 / 209
        luma = np.full(count, 255)
        score = rng.integers(lo, hi + 1, size=count) * 209 // 255 + 1
        p = _with_scores(pays[0], vd, 1, score, luma)
        p = _with_scores(p, vd, 0, score, luma)
        out.append((f"forced class {target}", vd, p, {}))
    luma = rng.integers(0, 256, size=count)
    score = rng.integers(0, 1 << 24, size=count)  # scores above 8.4 M saturate score * 255
    p = _with_scores(_with_scores(pays[1], vd, 0, score[::-1], luma), vd, 1, score, luma[::-1])
    for kw in ({}, {"gamma": 1.0}, {"gamma": 2.2, "blocks": 50, "scene": 8000}, {"gamma": 0.5, "zero": 0},
               {"blocks": 0}, {"blocks": 100, "m1": 0, "m2": 0}):
        out.append((f"random {kw}", vd, p, kw))
    vd1, pays1 = _payloads(aopt="{vectors:1,block:{w:8,overlap:0},main:{search:{type:2,distance:4}}}", seed=52)
    out.append(("previous set only", vd1, pays1[0], {}))
    vd3, pays3 = _payloads(w=160, h=96, aopt="{block:{w:32,overlap:3}}", seed=53)
    out.append(("block 32", vd3, pays3[0], {"gamma": 1.8}))
    none = pays[0].copy()
    none[8:12] = 0  # flags 0: no vector set at all -> class 3
    out.append(("no vector set", [vd[0], 0] + list(vd[2:]), none, {}))
    bad = pays[0].copy()
    bad[8] ^= 3
    out.append(("undecodable", vd, bad, {}))
    return out


CASES = _cases()


@pytest.mark.parametrize("case", range(len(CASES)))
def test_oracle_scene_class_matches_python(case):
    name, vd, p, kw = CASES[case]
    got = orc.scene_class(vd, p, **kw)
    if name == "undecodable":
        assert got == -1
        return
    assert got == _py_scene(vd, p, **kw), name
    if name.startswith("forced class"):
        assert got == int(name[-1])
    if name == "no vector set":
        assert got == 3


@pytest.mark.gpu
def test_device_scene_class_matches_oracle():
    import torch

    import svpflow_b200 as sv

    groups = {}
    for name, vd, p, kw in CASES:
        groups.setdefault((tuple(vd), tuple(sorted(kw.items()))), []).append((name, p))
    for (vd, kw), items in groups.items():
        vd, kw = list(vd), dict(kw)
        pays = np.stack([p for _, p in items])
        src = torch.from_numpy(pays).cuda()
        classes = torch.full((len(items),), 99, dtype=torch.int32, device="cuda")
        status = torch.full((len(items),), 9, dtype=torch.int32, device="cuda")
        sv.scene_class_device(vd, src.data_ptr(), pays.shape[1], len(items), classes.data_ptr(), status.data_ptr(),
                              **kw)
        torch.cuda.synchronize()
        got, st = classes.cpu().numpy(), status.cpu().numpy()
        for i, (name, p) in enumerate(items):
            want = orc.scene_class(vd, p, **kw)
            assert got[i] == want, f"{name}: {got[i]} != {want}"
            assert st[i] == (1 if want < 0 else 0), name
