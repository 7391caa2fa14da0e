"""The C ABI library on CPU: it loads, exports every declared symbol, and its host-side
option handling (opt-string parser, SuperOpts/AnalyseOpts derivation, vdata header) agrees
with the oracle's restatement. No compute call is made here (no GPU in this container)."""
import ctypes
import os
import re

import pytest

from oracle import oracle as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _sv():
    import svpflow_b200 as sv

    return sv


def test_library_exports_every_declared_symbol():
    sv = _sv()
    hdr = open(os.path.join(ROOT, "include", "svpflow_b200.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    names = set(re.findall(r"\b(svpf_[a-z0-9_]+)\s*\(", hdr))
    assert len(names) >= 25
    lib = ctypes.CDLL(sv.LIB_PATH)
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_reference_version():
    assert _sv().lib().svpf_reference_version() == 1174405393


OPTS = [
    None, "", "{}", "{pel:1}", "{pel:4, gpu:0}", "{ \"pel\" : 2 , gpu: 2 }",
    "// comment\n{pel:1}", "/* c */ {pel:4}", "{pel:1, pel:4}",         # last duplicate wins
    "{pel:2.9}", "{pel:true}", "{pel:null}", "{pel:\"4\"}",              # int_at truncation / bool / null / string
    "{full:0, pel:1}", "{full:[], pel:1}", "{full:\"x\", pel:1}",
    "{pel:1e0}", "{pel:-.5e1}", "{pel:4} trailing", "[1,2]", "12", "{pel:",   # parse errors -> defaults
    "{scale:{up:2,down:2},gpu:0}",
]


@pytest.mark.parametrize("opt", OPTS)
def test_super_options_match_oracle(opt):
    sv = _sv()
    try:
        so = orc.super_opts(320, 240, opt)
    except ValueError as e:
        with pytest.raises(ValueError, match=re.escape(str(e))):
            sv.Super(320, 240, opt)
        return
    sb = sv.Super(320, 240, opt)
    assert sb.sdata == orc.sdata(so)
    assert sb.super_height == orc.super_height(so)
    assert sb.output_len() == orc.super_output_len(so)


AOPTS = [
    None, "{}", "{vectors:1}", "{vectors:2,block:{w:8,h:4,overlap:1}}", "{block:{w:32,overlap:0}}",
    "{delta:3}", "{special:{delta:2},delta:5}", "{main:{penalty:{lambda:2.5,lsad:100,plevel:2,pnew:-30}}}",
    "{penalty:{lambda:1,pzero:7}}", "{main:{search:{type:2,distance:-6,coarse:{type:4,distance:3,bad:{sad:5,range:7}}}}}",
    "{search:{satd:true,coarse:{satd:false}}}", "{main:{search:{coarse:{satd:false}}}}", "{main:{levels:2}}",
    "{main:{levels:40}}", "{refine:[{thsad:200,search:{type:2,distance:3,satd:true}}]}", "{refine:[]}",
    "{refine:[5]}", "{sort:false}", "{main:{search:{sort:0}}}", "{block:{w:16,overlap:3},main:{search:{type:3,distance:16,satd:true}}}",
    "{vectors:4}", "{block:{w:7}}", "{block:{overlap:9}}",
]


@pytest.mark.parametrize("opt", AOPTS)
def test_analyse_options_match_oracle(opt):
    sv = _sv()
    so = orc.super_opts(640, 360, "{pel:2}")
    sd = orc.sdata(so)
    try:
        ao = orc.analyse_opts(sd, opt, None, 640, 360)
    except ValueError as e:
        with pytest.raises(ValueError, match=re.escape(str(e))):
            sv.Analyse(sd, opt, 640, 360)
        return
    try:
        an = sv.Analyse(sd, opt, 640, 360)
    except sv.SvpfError as e:  # options the device path refuses must be the documented ones
        assert e.code == sv.SVPF_EUNSUP and ao.has_refine_thsad
        return
    assert an.vector_header() == orc.vdata_header(ao)
    assert an.payload_len() == orc.payload_len(ao)
    assert an.delta == ao.delta


def test_invalid_sdata_is_an_error():
    sv = _sv()
    with pytest.raises(ValueError, match="SVAnalyse: invalid super clip params"):
        sv.Analyse(0, "{}", 640, 360)


def test_portable_constructors_match_oracle():
    sv = _sv()
    for (w, h, pel) in [(640, 360, 1), (320, 240, 2), (256, 144, 4)]:
        sb = sv.SuperBuilder(w, h, pel)
        so = orc.super_opts_portable(w, h, pel)
        assert sb.sdata == orc.sdata(so) and sb.levels == so.levels
        for (bw, bh, om, vec) in [(16, 16, 2, 3), (8, 8, 0, 1), (32, 16, 3, 2)]:
            an = sv.Analyser(sb, bw, bh, om, vec)
            ao = orc.analyser_portable(so, bw, bh, om, vec)
            assert an.vector_header() == orc.vdata_header(ao)
    with pytest.raises(ValueError, match="pel must be 1, 2 or 4"):
        sv.SuperBuilder(64, 64, 3)
    with pytest.raises(ValueError, match="dimensions must be positive and even"):
        sv.SuperBuilder(65, 64, 2)
    with pytest.raises(ValueError, match="block dimensions must be 4, 8, 16 or 32"):
        sv.Analyser(sv.SuperBuilder(64, 64, 2), 12, 16, 2, 3)


def test_compute_entry_points_fail_loudly_without_a_gpu():
    """No CPU fallback: with no CUDA device every compute call is an error (this container
    has none; on a GPU machine the GPU suite covers these calls)."""
    import numpy as np

    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a CUDA device is present")
    except ImportError:
        pass
    sv = _sv()
    sb = sv.Super(64, 48, "{pel:2}")
    an = sv.Analyse(sb.sdata, "{block:{w:8}}", 64, 48)
    frames = np.zeros((2, sb.source_len()), np.uint8)
    vd = an.vector_header()
    cfg = dict(width=64, height=48, block_w=8, block_h=8, origin_x=4, origin_y=4, grid_w=8, grid_h=6, source_step=1)
    calls = (lambda: sb.build_many(frames), lambda: an.analyse_clip(sb, frames),
             lambda: sv.Batch([(sb, an, 2)]), lambda: sv.Server(1 << 30),
             # the payload consumers refuse before touching their (here dummy) device pointers
             lambda: sv.vector_planes_device(vd, 16, 4096, 1, 64, 48, 16, 16),
             lambda: sv.render_masks_device(vd, 16, 4096, 1, 128, 16, 16, 16),
             lambda: sv.scene_class_device(vd, 16, 4096, 1, 16, 16),
             lambda: sv.render_warp_device(cfg, 128, False, True, [16] * 3, [64, 32, 32], [1] * 3, 0, 16, 16,
                                           [16] * 3, [64, 32, 32]))
    for call in calls:
        with pytest.raises(sv.SvpfError, match="no CUDA device") as e:
            call()
        assert e.value.code == sv.SVPF_ECUDA


@pytest.mark.parametrize("lang,std", [("c", "c99"), ("c++", "c++11")])
def test_header_is_plain_c_and_cxx(lang, std):
    """include/svpflow_b200.h is the C ABI a foreign host binds: it must compile on its own as strict
    C99 and C++11 (no torch or CUDA types in the signatures), warning-free."""
    import shutil
    import subprocess

    cc = shutil.which("gcc" if lang == "c" else "g++")
    if cc is None:
        pytest.skip("no host compiler")
    header = os.path.join(ROOT, "include", "svpflow_b200.h")
    r = subprocess.run([cc, "-x", lang, f"-std={std}", "-Wall", "-Wextra", "-pedantic", "-Werror", "-fsyntax-only",
                        header], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    src = open(header).read()
    assert "torch" not in src and "cuda_runtime" not in src and "at::" not in src


def test_lookahead_mode_bits():
    """svpf_analyser_set_lookahead takes the bit set 0..7 (1 level 0, 2 the coarser levels, 4
    level 0 spread over the GPU) and rejects anything else; setting it needs no GPU."""
    import svpflow_b200 as sv

    sb = sv.Super(64, 48, "{pel:2}")
    an = sv.Analyse(sb.sdata, "{}", 64, 48)
    for mode in range(8):
        an.set_lookahead(mode)
    an.set_lookahead(True)
    an.set_lookahead(False)
    for bad in (-1, 8):
        with pytest.raises(ValueError, match="look-ahead mode must be 0..7"):
            an.set_lookahead(bad)
