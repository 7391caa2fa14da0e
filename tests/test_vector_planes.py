"""Consumers of the payload (svpflow-core metadata.rs decode_vectors, renderer.rs vector_planes):
the oracle against a direct decoding of the payload bytes (CPU), and the device kernel against the
oracle on real Analyse payloads (GPU, bit-exact), including payloads that do not decode."""
import numpy as np
import pytest

from oracle import oracle as orc
from payload import decode


def _payloads(w=160, h=96, n=3, sopt="{pel:2}", aopt="{block:{w:16,overlap:2},main:{search:{type:3,distance:8}}}"):
    from svpflow_b200.synth import make_clip

    clip = make_clip(w, h, n, seed=31, motion=8, objects=2, object_motion=12)
    so = orc.super_opts(w, h, sopt)
    ao = orc.analyse_opts(orc.sdata(so), aopt, None, w, h)
    sup = orc.build_super_many(so, clip)
    return orc.vdata_header(ao), orc.analyse_clip(ao, so, sup, 0, n), (w, h)


def test_oracle_planes_follow_the_payload():
    vd, pays, (w, h) = _payloads()
    mw, mh = orc.vector_grid(vd)
    bw, ox, gw = vd[2], vd[9], vd[11]
    assert mw == gw + ((bw - ox) * gw + ox < w)
    for p in pays:
        planes = orc.vector_planes(vd, p, w, h, raw=True)
        d = decode(p)
        for which, key in ((0, "previous"), (1, "current")):
            dx = np.asarray(d[key]["dx"]).reshape(vd[12], vd[11])
            dy = np.asarray(d[key]["dy"]).reshape(vd[12], vd[11])
            ys = np.minimum(np.arange(mh), vd[12] - 1)[:, None]
            xs = np.minimum(np.arange(mw), vd[11] - 1)[None, :]
            ex, ey = dx[ys, xs].astype(int), dy[ys, xs].astype(int)
            big = (np.abs(ex) > 1023) | (np.abs(ey) > 1023)
            assert (planes[2 * which] == np.where(big, 1024, ex + 1024)).all()
            assert (planes[2 * which + 1] == np.where(big, 1024, ey + 1024)).all()
    bad = pays[0].copy()
    bad[4] ^= 1  # magic
    assert orc.vector_planes(vd, bad, w, h) is None


def _clamp_to_frame(v, pos, block, frame):  # renderer.rs clamp_to_frame
    if v + pos < 0:
        return -pos
    if v + block + pos > frame:
        return max(frame - block - pos, 0)
    return v


@pytest.mark.parametrize("frame", [(160, 96), (120, 70)])
def test_oracle_planes_clamp_to_the_frame(frame):
    # raw = False: each vector is clamped so its block stays inside the frame, at the block's
    # position x * (block - overlap); vectors beyond +-1023 become the neutral 1024
    vd, pays, _ = _payloads()
    mw, mh = orc.vector_grid(vd)
    bw, bh, stx, sty = vd[2], vd[3], vd[2] - vd[9], vd[3] - vd[10]
    rng = np.random.default_rng(5)
    p = pays[1].copy()
    count = vd[11] * vd[12]
    words = p[0x44: 0x44 + 8 * count].view(np.uint32).reshape(count, 2).copy()
    dx, dy = rng.integers(-1100, 1100, size=count), rng.integers(-1100, 1100, size=count)
    words[:, 0] = (dx.astype(np.int64).astype(np.uint32) << 16) | (dy.astype(np.int64) & 0xFFFF).astype(np.uint32)
    p[0x44: 0x44 + 8 * count] = words.reshape(-1).view(np.uint8)
    got = orc.vector_planes(vd, p, frame[0], frame[1])
    d = decode(p)["previous"]
    for y in range(mh):
        for x in range(mw):
            k = min(y, vd[12] - 1) * vd[11] + min(x, vd[11] - 1)
            vx, vy = int(d["dx"][k]), int(d["dy"][k])
            if abs(vx) > 1023 or abs(vy) > 1023:
                want = (1024, 1024)
            else:
                want = (_clamp_to_frame(vx, x * stx, bw, frame[0]) + 1024, _clamp_to_frame(vy, y * sty, bh, frame[1]) + 1024)
            assert (got[0][y, x], got[1][y, x]) == want, (x, y)


@pytest.mark.gpu
@pytest.mark.parametrize("aopt", ["{block:{w:16,overlap:2},main:{search:{type:3,distance:8}}}",
                                  "{vectors:1,block:{w:8,overlap:0},main:{search:{type:2,distance:4}}}",
                                  "{vectors:2,block:{w:32,overlap:3}}"])
def test_device_planes_match_oracle(aopt):
    import torch

    import svpflow_b200 as sv

    vd, pays, (w, h) = _payloads(aopt=aopt)
    n = len(pays)
    mw, mh = sv.vector_grid(vd)
    bad = pays.copy()
    bad[1, 8] ^= 3  # flags word: this payload must not decode
    for frame in ((w, h), (w - 40, h - 20)):
        for raw in (False, True):
            src = torch.from_numpy(bad).cuda()
            planes = torch.full((n, 4 * mw * mh), 7, dtype=torch.int16, device="cuda")
            status = torch.zeros(n, dtype=torch.int32, device="cuda")
            sv.vector_planes_device(vd, src.data_ptr(), pays.shape[1], n, frame[0], frame[1], planes.data_ptr(),
                                    status.data_ptr(), raw=raw)
            torch.cuda.synchronize()
            got = planes.cpu().numpy().view(np.uint16).reshape(n, 4, mh, mw)
            st = status.cpu().numpy()
            for i in range(n):
                want = orc.vector_planes(vd, bad[i], frame[0], frame[1], raw=raw)
                if want is None:
                    assert st[i] == 1
                else:
                    assert st[i] == 0 and np.array_equal(got[i], want), f"payload {i}, frame {frame}, raw {raw}"
