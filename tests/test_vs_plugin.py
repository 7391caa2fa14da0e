"""The VapourSynth plugin (libsvpflow1_vs.so) against a stand-in frame server (tests/vsfake.py):
exports, plugin identity and registrations (crates/svpflow1/src/abi.rs), argument errors
and published values of the Super and Analyse filters (super_filter.rs, analyse_filter.rs)
on the CPU; on the GPU, frames through getFrame compared byte for byte with the oracle run
at the same row pitches."""
import ctypes
import os

import numpy as np
import pytest

from oracle import oracle as orc
from vsfake import Plugin, Server

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
VS_LIB = os.path.join(ROOT, "open-svpflow_b200", "lib", "libsvpflow1_vs.so")


@pytest.fixture()
def vs():
    srv = Server(align=64)
    return srv, Plugin(VS_LIB, srv)


def _clip(srv, w=128, h=96, n=4, seed=5):
    from svpflow_b200.synth import make_clip

    frames = make_clip(w, h, n, seed=seed, motion=5, objects=2, object_motion=8)
    return frames, srv.source_clip(frames, w, h)


def test_exports_and_registration(vs):
    srv, pl = vs
    assert pl.lib.svpGetVersion() == 1174405393
    assert pl.config_calls == [("com.svp-team.flow1", "svp1", "SVPFlow1", 0x30002, 1, 0x1234)]
    assert {k: v[0] for k, v in pl.functions.items()} == {
        "Super": "clip:clip;opt:data", "Analyse": "clip:clip;sdata:int;src:clip;opt:data"}
    # no config callback: nothing is registered; config but no register: identity only
    calls = []
    from vsfake import CONFIG

    cfg = CONFIG(lambda *a: calls.append(a))
    pl.lib.VapourSynthPluginInit(None, None, None)
    pl.lib.VapourSynthPluginInit(ctypes.cast(cfg, ctypes.c_void_p), None, None)
    assert len(calls) == 1


def test_super_arguments_and_published_values(vs):
    srv, pl = vs
    out, _ = pl.invoke("Super", {})
    assert out["_error"] == "SVSuper: clip is required"
    frames, clip = _clip(srv)
    out, _ = pl.invoke("Super", {"clip": clip, "opt": "{pel:3}"})
    assert out["_error"] == "SVSuper: pel has to be 1 or 2 or 4"
    for opt in (None, "{pel:1}", "{pel:4, gpu:0}", "{pel:2", ""):
        args = {"clip": clip} if opt is None else {"clip": clip, "opt": opt}
        out, _ = pl.invoke("Super", args)
        assert "_error" not in out
        so = orc.super_opts(128, 96, opt if opt else None)
        assert out["data"] == ("int", orc.sdata(so))
        node = srv.objs[out["clip"][1]]
        assert node.name == "SVSuper" and node.mode == 100
        assert (node.vi.width, node.vi.height, node.vi.num_frames) == (128, orc.super_height(so), 4)
        assert node.vi.format == srv.objs[clip].vi.format


def test_analyse_arguments_and_published_values(vs):
    srv, pl = vs
    frames, clip = _clip(srv)
    sup, _ = pl.invoke("Super", {"clip": clip, "opt": "{pel:2}"})
    snode, sdata = sup["clip"][1], sup["data"][1]
    from vsfake import NodeRef

    snode = NodeRef(snode)
    for args, msg in [({}, "SVAnalyse: clip (super) required"),
                      ({"clip": snode}, "SVAnalyse: src required"),
                      ({"clip": snode, "src": clip}, "SVAnalyse: sdata required"),
                      ({"clip": snode, "src": clip, "sdata": sdata, "opt": "{vectors:0}"},
                       "SVAnalyse: vectors must be 1, 2 or 3"),
                      ({"clip": snode, "src": clip, "sdata": 0}, "SVAnalyse: invalid super clip params")]:
        out, _ = pl.invoke("Analyse", args)
        assert out["_error"] == msg
    opt = "{block:{w:16,overlap:2},main:{search:{type:3,distance:6,satd:true}}}"
    out, _ = pl.invoke("Analyse", {"clip": snode, "src": clip, "sdata": sdata, "opt": opt})
    assert "_error" not in out
    ao = orc.analyse_opts(sdata, opt, None, 128, 96)
    hdr = (ctypes.c_int32 * 16).from_address(out["data"][1])  # `data` is the header's address
    assert list(hdr) == orc.vdata_header(ao)
    node = srv.objs[out["clip"][1]]
    assert node.name == "SVAnalyse" and node.mode == 100
    assert (node.vi.width, node.vi.height, node.vi.num_frames) == (orc.payload_len(ao), 1, 4)
    assert node.vi.format == ctypes.addressof(srv.fmt_gray)
    assert (node.vi.fps_num, node.vi.fps_den) == (30000, 1001)
    srv.gray_preset = False  # no Gray8 preset: the super clip's format stands in
    out, _ = pl.invoke("Analyse", {"clip": snode, "src": clip, "sdata": sdata})
    assert srv.objs[out["clip"][1]].vi.format == srv.objs[snode].vi.format


CASES = [  # (w, h, frames, align, super opt, analyse opt)
    (128, 96, 4, 64, "{pel:2}", "{block:{w:16,overlap:2},main:{search:{type:3,distance:6,satd:true}}}"),
    (160, 96, 3, 32, "{pel:1}", "{block:{w:8,overlap:0},main:{search:{type:2,distance:2}}}"),
    (96, 64, 3, 128, "{pel:4}", "{delta:2,block:{w:8,overlap:3},main:{search:{type:4,distance:2,satd:true}}}"),
    (130, 70, 3, 64, "{pel:2,gpu:0}", "{vectors:1,block:{w:16,overlap:1}}"),
]


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=[f"{c[0]}x{c[1]}_a{c[3]}_{c[4]}" for c in CASES])
def test_frames_match_oracle_at_frame_server_pitches(case):
    w, h, n, align, sopt, aopt = case
    srv = Server(align=align)
    pl = Plugin(VS_LIB, srv)
    frames, clip = _clip(srv, w, h, n, seed=w + h)
    sup, _ = pl.invoke("Super", {"clip": clip, "opt": sopt})
    so = orc.super_opts(w, h, sopt)
    snode = sup["clip"][1]
    from vsfake import NodeRef

    ana, _ = pl.invoke("Analyse", {"clip": NodeRef(snode), "src": clip, "sdata": sup["data"][1], "opt": aopt})
    ao = orc.analyse_opts(orc.sdata(so), aopt, None, w, h)
    want_sup = []
    for i in range(n):
        fr = srv.frame(srv.get_frame(snode, i))
        ys, cs = fr.strides[0], fr.strides[1]
        got = np.concatenate([fr.planes[p][: fr.strides[p] * fr.rows[p]] for p in range(3)])
        want = orc.build_super_strided(so, frames[i], ys, cs)
        assert np.array_equal(got, want), f"super frame {i} differs (pitches {ys}/{cs})"
        want_sup.append(want)
    pl_len = orc.payload_len(ao)
    for i in range(n):
        fr = srv.frame(srv.get_frame(ana["clip"][1], i))
        row = fr.planes[0][: fr.strides[0]]
        j = min(i + max(ao.delta, 1), n - 1)
        want = orc.analyse_strided(ao, want_sup[i], want_sup[j], ys, cs)
        assert np.array_equal(row[:pl_len], want), f"payload of frame {i} differs"
        assert not row[pl_len:].any()  # zero-padded to the row pitch
    srv.free_filter(ana["clip"][1])
    srv.free_filter(snode)
