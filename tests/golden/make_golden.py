"""Generates tests/golden/oracle_digests.json: SHA-256 digests of the oracle's super frames
and Analyse payloads on seeded synthetic clips.

These digests freeze the oracle (oracle/svpf_oracle.c) after it was checked against the
independent Python restatement; they are a regression guard for both the oracle and the
GPU path, not outputs of the Rust reference (which cannot run in this image).

    python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "open-svpflow_b200"), ROOT]

from oracle import oracle as orc  # noqa: E402
from svpflow_b200.synth import make_clip  # noqa: E402

# name: (w, h, frames, seed, synth kwargs, super opt, analyse opt)
CASES = {
    "cfg1_640x360_pel1_hex2_sad": (640, 360, 4, 1, dict(motion=8, objects=4, object_motion=16), "{pel:1}",
                                   "{block:{w:16,overlap:0},main:{search:{type:2,distance:2,satd:false,coarse:{satd:false}}}}"),
    "cfg2_shape_320x180_pel2_umh16_satd": (320, 180, 3, 2, dict(motion=12, objects=4, object_motion=24), "{pel:2}",
                                           "{block:{w:16,overlap:3},main:{search:{type:3,distance:16,satd:true}}}"),
    "cfg3_shape_256x144_pel4_exh_blk8": (256, 144, 3, 3, dict(motion=16, objects=3, object_motion=20), "{pel:4}",
                                         "{block:{w:8,overlap:3},main:{search:{type:4,distance:8,satd:true,coarse:{type:2}}}}"),
    "defaults_192x128_pel2": (192, 128, 3, 4, dict(motion=6, objects=2, object_motion=8), "{pel:2}", "{}"),
    "bicubic_blk32_192x128": (192, 128, 2, 5, dict(motion=6, objects=2, object_motion=8), "{pel:2,gpu:0}",
                              "{block:{w:32,overlap:1},main:{search:{type:3,distance:8}}}"),
    "blk4_vectors1_128x96": (128, 96, 3, 6, dict(motion=4, objects=2, object_motion=6), "{pel:2}",
                             "{vectors:1,block:{w:4,overlap:0},main:{search:{type:2,distance:4}}}"),
}


def digest(a) -> str:
    return hashlib.sha256(bytes(a)).hexdigest()


def compute(name):
    w, h, n, seed, kw, sopt, aopt = CASES[name]
    clip = make_clip(w, h, n, seed=seed, **kw)
    so = orc.super_opts(w, h, sopt)
    ao = orc.analyse_opts(orc.sdata(so), aopt, None, w, h)
    supers = orc.build_super_many(so, clip, 4)
    pays = orc.analyse_clip(ao, so, supers, 0, n, 4)
    return {"super": [digest(supers[i]) for i in range(n)], "payload": [digest(pays[i]) for i in range(n)]}


def main():
    out = {"note": "oracle digests (regression guard; not outputs of the Rust reference)", "cases": {}}
    for name in CASES:
        out["cases"][name] = compute(name)
        print(name, "done", flush=True)
    with open(os.path.join(HERE, "oracle_digests.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
