"""Generates tests/golden/consumer_digests.json: SHA-256 digests of the oracle's payload consumers
(vector planes, mask planes, scene classes, rendered planes of algorithms 2, 13, 21 and 23) on the
payloads of seeded synthetic clips.

Like oracle_digests.json these freeze the oracle after it was checked against the independent Python
restatements (tests/test_vector_planes.py, test_masks.py, test_scene.py, test_render.py); they are a
regression guard, not outputs of the Rust reference (which cannot run in this image).

    python tests/golden/make_consumer_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "open-svpflow_b200"), ROOT]

from oracle import oracle as orc  # noqa: E402
from svpflow_b200.synth import make_clip  # noqa: E402

# name: (w, h, frames, seed, synth kwargs, super opt, analyse opt)
CASES = {
    "umh16_320x180": (320, 180, 4, 21, dict(motion=10, objects=3, object_motion=16), "{pel:2}",
                      "{block:{w:16,overlap:3},main:{search:{type:3,distance:16,satd:true}}}"),
    "blk8_ov2_256x144": (256, 144, 4, 22, dict(motion=6, objects=3, object_motion=10), "{pel:2}",
                         "{block:{w:8,overlap:2},main:{search:{type:2,distance:4}}}"),
}
PHASE, COVER, SCALE = 96, 100, 0.0256


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def compute(name):
    w, h, n, seed, kw, sopt, aopt = CASES[name]
    clip = make_clip(w, h, n, seed=seed, **kw)
    so = orc.super_opts(w, h, sopt)
    ao = orc.analyse_opts(orc.sdata(so), aopt, None, w, h)
    supers = orc.build_super_many(so, clip)
    pays = orc.analyse_clip(ao, so, supers, 0, n)
    vd = orc.vdata_header(ao)
    mw, mh = orc.vector_grid(vd)
    planes = [orc.vector_planes(vd, pays[f], w, h) for f in range(n)]
    masks = [orc.render_masks(vd, pays[f], PHASE, COVER, SCALE, sharp) for f in range(n) for sharp in (1.0, 0.6)]
    scenes = [orc.scene_class(vd, pays[f], **kw2) for f in range(n) for kw2 in ({}, {"gamma": 1.0, "blocks": 50})]
    # renders of frame 1 from the pel-2 super frames, SmoothFps's configuration (effective block)
    hs = orc.super_height(so)
    cfg = dict(width=w, height=h, block_w=vd[2] - vd[9], block_h=vd[3] - vd[10], origin_x=vd[2] // 2,
               origin_y=vd[3] // 2, grid_w=mw, grid_h=mh, chroma_y_div=2, source_step=2)
    offs = [0, w * hs, w * hs + (w // 2) * (hs // 2)]
    lens = [w * hs, (w // 2) * (hs // 2), (w // 2) * (hs // 2)]
    f = 1
    mp, om = planes[f], orc.render_masks(vd, pays[f], PHASE, COVER, SCALE)
    tl = orc.render_threshold_limit(PHASE, SCALE)
    _, lut = orc.render_luts(PHASE)
    renders = []
    for p in range(3):
        pw, ph = (w // 2, h // 2) if p else (w, h)
        srcs = [supers[f][offs[p]: offs[p] + lens[p]], supers[f + 1][offs[p]: offs[p] + lens[p]]]
        renders.append(orc.render_warp_plane(cfg, p > 0, True, lut, srcs[0], pw, pw * ph, 1, mp[0], mp[1], pw, ph,
                                             mask=om[3]))
        args = (srcs, [pw, pw], [pw * ph, pw * ph], 1, (mp[0], mp[1]), (mp[2], mp[3]), pw, ph)
        renders.append(orc.render_dual_plane(cfg, p > 0, True, False, 13, PHASE, *args))
        renders.append(orc.render_dual_plane(cfg, p > 0, True, False, 21, PHASE, *args, (om[0], om[1]), om[4], tl))
        motions = [(mp[0], mp[1]), (mp[2], mp[3]), (planes[f + 1][0], planes[f + 1][1]),
                   (planes[f - 1][2], planes[f - 1][3])]
        renders.append(orc.render_mode23_plane(cfg, p > 0, True, PHASE, srcs, [pw, pw], [pw * ph, pw * ph], 1,
                                               motions, (om[0], om[1]), om[4], pw, ph))
    return {"vector_planes": [digest(x) for x in planes], "mask_planes": [digest(x) for x in masks],
            "scene_classes": [int(c) for c in scenes], "renders": [digest(x) for x in renders]}


def main():
    out = {"note": "oracle digests of the payload consumers (regression guard; not outputs of the Rust reference)",
           "phase": PHASE, "cover": COVER, "area_scale": SCALE, "cases": {}}
    for name in CASES:
        out["cases"][name] = compute(name)
        print(name, "done", flush=True)
    with open(os.path.join(HERE, "consumer_digests.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
