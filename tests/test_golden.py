"""Frozen digests (tests/golden/oracle_digests.json, made by tests/golden/make_golden.py):
the oracle must keep producing them (CPU), and the GPU path must produce the same bytes. The
payload consumers' digests (tests/golden/consumer_digests.json, made by
tests/golden/make_consumer_golden.py) guard the oracle's vector planes, mask planes, scene classes
and renders the same way."""
import hashlib
import json
import os

import numpy as np
import pytest

from golden import make_consumer_golden as consumers
from golden import make_golden16 as golden16
from golden.make_golden import CASES, compute

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "oracle_digests.json")))["cases"]
CGOLD = json.load(open(os.path.join(HERE, "golden", "consumer_digests.json")))["cases"]
GOLD16 = json.load(open(os.path.join(HERE, "golden", "oracle16_digests.json")))["cases"]


@pytest.mark.parametrize("name", sorted(golden16.CASES))
def test_oracle16_matches_frozen_digests(name):
    assert golden16.compute(name) == GOLD16[name]


@pytest.mark.parametrize("name", sorted(consumers.CASES))
def test_oracle_consumers_match_frozen_digests(name):
    assert consumers.compute(name) == CGOLD[name]


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_frozen_digests(name):
    assert compute(name) == GOLD[name]


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_gpu_matches_frozen_digests(name):
    import svpflow_b200 as sv
    from svpflow_b200.synth import make_clip

    w, h, n, seed, kw, sopt, aopt = CASES[name]
    clip = make_clip(w, h, n, seed=seed, **kw)
    sb = sv.Super(w, h, sopt)
    an = sv.Analyse(sb.sdata, aopt, w, h)
    supers = sb.build_many(clip)
    pays = an.analyse_clip(sb, clip)
    d = lambda a: hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()
    assert [d(supers[i]) for i in range(n)] == GOLD[name]["super"]
    assert [d(pays[i]) for i in range(n)] == GOLD[name]["payload"]
