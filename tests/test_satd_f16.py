"""8-bit SATD in f16x2 (csrc/analyse_body.cuh, satd_rows_h): a sample s becomes the half
1024 + s, differences and the Hadamard butterflies run in IEEE half precision (round to nearest,
as add.rn.f16x2), |x| clears the sign, the last stage takes max(|a|, |b|) (|a + b| + |a - b| =
2 max), and the maxima are summed in f32. Every value is an integer of magnitude <= 8 * 255 =
2040, which halves hold exactly, so the result equals the integer transform's. Restated here in
numpy float16 on random tiles and on the extreme ones (0 / 255 patterns that maximise every
stage), and compared with the same transform in int64. CPU only; tolerance zero."""
import numpy as np


def _satd_stages(d01, d23, add, sub, absf, maxf, acc0):
    """satd_rows / satd_rows_h: d01[r] = (d0, d1), d23[r] = (d2, d3) as pairs of lanes."""
    h0, h1 = [], []
    for r in range(4):
        c = add(d01[r], d23[r])
        e = sub(d01[r], d23[r])
        p = np.stack([c[..., 0], e[..., 0]], axis=-1)  # byte_perm 0x5410: c.lo, e.lo
        q = np.stack([c[..., 1], e[..., 1]], axis=-1)  # byte_perm 0x7632: c.hi, e.hi
        h0.append(add(p, q))
        h1.append(sub(p, q))
    acc = acc0
    for h in (h0, h1):
        a0, a1 = add(h[0], h[1]), sub(h[0], h[1])
        a2, a3 = add(h[2], h[3]), sub(h[2], h[3])
        for m in (maxf(absf(a0), absf(a2)), maxf(absf(a1), absf(a3))):
            acc = acc + m[..., 0].astype(acc.dtype) + m[..., 1].astype(acc.dtype)
    return acc


def satd_int(src, ref):
    d = src.astype(np.int64) - ref.astype(np.int64)  # (..., 4 rows, 4 samples)
    d01 = [d[..., r, 0:2] for r in range(4)]
    d23 = [d[..., r, 2:4] for r in range(4)]
    acc = _satd_stages(d01, d23, np.add, np.subtract, np.abs, np.maximum, np.zeros(d.shape[:-2], np.int64))
    return 2 * acc


def satd_f16(src, ref):
    bias = lambda s: (np.float16(1024) + s.astype(np.float16)).astype(np.float16)  # exact: 1024 + s < 2048
    hs, hr = bias(src), bias(ref)
    assert np.array_equal(hs.astype(np.int64) - 1024, src.astype(np.int64))
    d = (hs - hr).astype(np.float16)
    d01 = [d[..., r, 0:2] for r in range(4)]
    d23 = [d[..., r, 2:4] for r in range(4)]
    f16 = lambda f: (lambda a, b: f(a, b).astype(np.float16))
    acc = _satd_stages(d01, d23, f16(np.add), f16(np.subtract), lambda a: np.abs(a).astype(np.float16),
                       f16(np.maximum), np.zeros(d.shape[:-2], np.float32))
    return 2 * acc.astype(np.int64)


def test_f16_satd_equals_integer_satd():
    rng = np.random.default_rng(11)
    src = rng.integers(0, 256, size=(200000, 4, 4), dtype=np.uint8)
    ref = rng.integers(0, 256, size=(200000, 4, 4), dtype=np.uint8)
    assert np.array_equal(satd_f16(src, ref), satd_int(src, ref))


def test_f16_satd_extreme_tiles():
    # every 0 / 255 pattern of the source tile against the complement and against flat tiles:
    # these reach the largest magnitude at every stage (|d| = 255, sums of up to 8 of them)
    bits = (np.arange(1 << 16)[:, None] >> np.arange(16)) & 1
    src = (bits * 255).astype(np.uint8).reshape(-1, 4, 4)
    for ref in (255 - src, np.zeros_like(src), np.full_like(src, 255)):
        got, want = satd_f16(src, ref), satd_int(src, ref)
        assert np.array_equal(got, want)
    # a flat difference has only the DC coefficient, 16 x 255
    assert satd_int(np.full((1, 4, 4), 255, np.uint8), np.zeros((1, 4, 4), np.uint8))[0] == 16 * 255


def test_integer_transform_is_the_oracles_satd():
    # the transform restated above is the oracle's 4x4 SATD (its restatement of the reference's
    # hadamard, analyse_search.rs:2305-2702), so the f16 form computes the reference's value
    from oracle import oracle as orc

    rng = np.random.default_rng(3)
    src = rng.integers(0, 256, size=(400, 4, 4), dtype=np.uint8)
    ref = rng.integers(0, 256, size=(400, 4, 4), dtype=np.uint8)
    want = [orc.hadamard4((src[i].astype(int) - ref[i].astype(int)).reshape(-1)) for i in range(len(src))]
    assert np.array_equal(satd_int(src, ref), np.array(want))
