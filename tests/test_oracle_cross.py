"""Differential test of the two restatements of the reference path (CPU): the C oracle
(oracle/svpf_oracle.c) and the independent pure-Python one (oracle/svpf_oracle_py.py) must
produce the same super frames and Analyse payloads, byte for byte, on small seeded clips; the
10-bit extension's 16-bit oracle build against the Python one with 10-bit samples likewise."""
import numpy as np
import pytest

from oracle import oracle as orc
from oracle import svpf_oracle_py as py
from svpflow_b200.synth import make_clip

# (w, h, seed, super opt, analyse opt)
CASES = [
    (64, 48, 1, "{pel:1}", "{block:{w:8,overlap:0},main:{search:{type:2,distance:2,satd:false,coarse:{satd:false}}}}"),
    (64, 48, 2, "{pel:2}", "{block:{w:8,overlap:2},main:{search:{type:3,distance:6,satd:true}}}"),
    (64, 48, 3, "{pel:4}", "{block:{w:8,overlap:3},main:{search:{type:4,distance:2,satd:true,coarse:{type:2}}}}"),
    (80, 48, 4, "{pel:2,gpu:0}", "{block:{w:16,overlap:2},main:{search:{type:2,distance:4}}}"),
    (64, 64, 5, "{pel:2}", "{vectors:1,block:{w:4,overlap:0},main:{search:{type:2,distance:3}}}"),
    (64, 48, 6, "{pel:2}", "{vectors:2,block:{w:8,overlap:1},main:{penalty:{pnew:-40},search:{type:3,distance:5}}}"),
    (96, 64, 7, "{pel:1}", "{block:{w:16,overlap:3},main:{search:{type:3,distance:8,coarse:{bad:{sad:1,range:3}}}}}"),
    (64, 48, 8, "{pel:2}", "{main:{search:{distance:0}}}"),
    # refine[0].thsad set: exact_recalculate onto half-size blocks (the second restatement's own copy)
    (64, 48, 9, "{pel:2}", "{refine:[{thsad:200,search:{type:2,distance:3,satd:true}}]}"),
    (96, 64, 10, "{pel:2}", "{block:{w:16,overlap:2},main:{search:{type:3,distance:6}},refine:[{thsad:50}]}"),
    (64, 48, 11, "{pel:4}", "{block:{w:8,overlap:0},refine:[{thsad:0,search:{type:4,distance:2}}]}"),
    (96, 64, 12, "{pel:1}", "{vectors:1,block:{w:32,overlap:1},refine:[{thsad:100,search:{type:3,distance:8}}]}"),
    (80, 48, 13, "{pel:2}", "{main:{search:{sort:false}},refine:[{thsad:20,search:{type:2,distance:2}}]}"),
    # coarse.distance < 0: the coarse levels' radius adapts to each block's activity (SAD / SATD forms)
    (96, 64, 14, "{pel:2}", "{block:{w:8,overlap:0},main:{search:{type:2,distance:2,coarse:{distance:-6}}}}"),
    (96, 64, 15, "{pel:2}", "{main:{search:{type:3,distance:4,coarse:{distance:-8,satd:false,type:3}}}}"),
]


@pytest.mark.parametrize("case", CASES, ids=[f"{c[0]}x{c[1]}_{c[3]}_{i}" for i, c in enumerate(CASES)])
def test_python_restatement_matches_c_oracle(case):
    w, h, seed, sopt, aopt = case
    clip = make_clip(w, h, 2, seed=seed, motion=5, objects=2, object_motion=7, noise=3)
    so = orc.super_opts(w, h, sopt)
    pso = py.super_from_opt(sopt, w, h)
    assert py.pack_data(pso) == orc.sdata(so)
    s_c = [orc.build_super(so, clip[i]) for i in range(2)]
    s_p = [py.build_super(pso, clip[i].tobytes()) for i in range(2)]
    for a, b in zip(s_c, s_p):
        assert a.tobytes() == b
    ao = orc.analyse_opts(orc.sdata(so), aopt, None, w, h)
    pay_c = orc.analyse(ao, so, s_c[1], s_c[0]).tobytes()
    pay_p = py.analyse(pso, aopt, s_p[1], s_p[0], w, h)
    assert len(pay_c) == len(pay_p)
    if pay_c != pay_p:
        a = np.frombuffer(pay_c, np.uint8)
        b = np.frombuffer(pay_p, np.uint8)
        i = int(np.nonzero(a != b)[0][0])
        pytest.fail(f"first differing byte {i} of {len(a)}: c={a[i]} py={b[i]}")


CASES16 = [  # the 10-bit extension: the same restatement with uint16 samples (clamps 1023, chroma 512)
    (64, 48, 21, "{pel:2}", "{block:{w:8,overlap:2},main:{search:{type:3,distance:6,satd:true}}}"),
    (64, 48, 22, "{pel:4}", "{block:{w:8,overlap:3},main:{search:{type:4,distance:2,satd:true,coarse:{type:2}}}}"),
    (80, 48, 23, "{pel:2,gpu:0}", "{block:{w:16,overlap:2},refine:[{thsad:40,search:{type:2,distance:2}}]}"),
]


@pytest.mark.parametrize("case", CASES16, ids=[f"{c[0]}x{c[1]}_{c[3]}_{i}" for i, c in enumerate(CASES16)])
def test_python_restatement_matches_c_oracle16(case):
    w, h, seed, sopt, aopt = case
    c8 = make_clip(w, h, 2, seed=seed, motion=5, objects=2, object_motion=7, noise=3)
    rng = np.random.default_rng(seed)
    clip = (c8.astype(np.uint16) << 2) | rng.integers(0, 4, size=c8.shape, dtype=np.uint16)
    so = orc.super_opts(w, h, sopt)
    pso = py.super_from_opt(sopt, w, h)
    s_c = orc.build_super_many16(so, clip)
    py.set_sample_bits(10)
    try:
        s_p = [py.build_super(pso, clip[i]) for i in range(2)]
        for i in range(2):
            assert np.array_equal(np.asarray(s_p[i], dtype=np.uint16), s_c[i]), f"super frame {i}"
        ao = orc.analyse_opts(orc.sdata(so), aopt, None, w, h)
        pay_c = orc.analyse_clip16(ao, so, s_c, 0, 1)[0].tobytes()
        pay_p = py.analyse(pso, aopt, s_p[0], s_p[1], w, h)
    finally:
        py.set_sample_bits(8)
    assert len(pay_c) == len(pay_p)
    if pay_c != pay_p:
        a = np.frombuffer(pay_c, np.uint8)
        b = np.frombuffer(pay_p, np.uint8)
        i = int(np.nonzero(a != b)[0][0])
        pytest.fail(f"first differing byte {i} of {len(a)}: c={a[i]} py={b[i]}")
