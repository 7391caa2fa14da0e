"""Generates tests/golden/oracle16_digests.json: SHA-256 digests of the 16-bit oracle's super frames
and payloads (this project's 10-bit extension: uint16 samples 0..1023) on seeded synthetic clips.

The extension has no reference behaviour; the oracle's -DOR_PX16 build defines it, and these digests
freeze that definition as a regression guard.

    python tests/golden/make_golden16.py
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
    "pel4_exh_blk8_256x144": (256, 144, 3, 31, dict(motion=10, objects=3, object_motion=14), "{pel:4}",
                              "{block:{w:8,overlap:3},main:{search:{type:4,distance:4,satd:true,coarse:{type:2}}}}"),
    "pel2_umh_blk16_320x180": (320, 180, 3, 32, dict(motion=12, objects=4, object_motion=20), "{pel:2}",
                               "{block:{w:16,overlap:2},main:{search:{type:3,distance:8,satd:true}}}"),
    "bicubic_refine_192x128": (192, 128, 2, 33, dict(motion=6, objects=2, object_motion=8), "{pel:2,gpu:0}",
                               "{refine:[{thsad:100,search:{type:2,distance:3,satd:true}}]}"),
}


def clip10(w, h, n, seed, kw):
    """The 8-bit synthetic recipe widened to 10 bits with seeded low bits."""
    c8 = make_clip(w, h, n, seed=seed, **kw)
    rng = np.random.default_rng(seed + 1)
    return (c8.astype(np.uint16) << 2) | rng.integers(0, 4, size=c8.shape, dtype=np.uint16)


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def compute(name):
    w, h, n, seed, kw, sopt, aopt = CASES[name]
    clip = clip10(w, h, n, seed, kw)
    so = orc.super_opts(w, h, sopt)
    ao = orc.analyse_opts(orc.sdata(so), aopt, None, w, h)
    supers = orc.build_super_many16(so, clip)
    pays = orc.analyse_clip16(ao, so, supers, 0, n)
    return {"super": [digest(supers[i]) for i in range(n)], "payload": [digest(pays[i]) for i in range(n)]}


def main():
    out = {"note": "16-bit oracle digests (the 10-bit extension's definition; regression guard)", "cases": {}}
    for name in CASES:
        out["cases"][name] = compute(name)
        print(name, "done", flush=True)
    with open(os.path.join(HERE, "oracle16_digests.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
