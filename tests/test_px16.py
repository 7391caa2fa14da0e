"""The 10-bit extension: uint16 samples (0..1023) through the same Super and Analyse.

The reference is 8-bit only, so this path has no reference behaviour to match; the oracle's
16-bit build (the same C restatement compiled with uint16 samples, clamps at 1023, chroma
default 512, payload luma byte = block mean >> 2) defines it and the GPU must equal it byte
for byte. CPU tests cover the host side; `gpu` tests the parity.
"""
import numpy as np
import pytest

from oracle import oracle as orc
from payload import first_difference


def _sv():
    import svpflow_b200 as sv

    return sv


def clip10(w, h, n, seed, **kw):
    """A seeded 10-bit clip: the 8-bit synthetic recipe widened to 10 bits with random low bits."""
    from svpflow_b200.synth import make_clip

    c8 = make_clip(w, h, n, seed=seed, **kw)
    rng = np.random.default_rng(seed + 1)
    return (c8.astype(np.uint16) << 2) | rng.integers(0, 4, size=c8.shape, dtype=np.uint16)


# ---------------------------------------------------------------- CPU

def test_oracle16_level0_is_the_source():
    w, h = 64, 48
    so = orc.super_opts(w, h, "{pel:2}")
    src = clip10(w, h, 1, seed=5)[0]
    sup = orc.build_super16(so, src)
    assert sup.dtype == np.uint16 and sup.max() <= 1023
    got_y = sup[: w * h].reshape(h, w)
    assert np.array_equal(got_y, src[: w * h].reshape(h, w))
    cw, ch = w // 2, h // 2
    u_off = w * orc.super_height(so)
    got_u = sup[u_off: u_off + cw * ch].reshape(ch, cw)
    assert np.array_equal(got_u, src[w * h: w * h + cw * ch].reshape(ch, cw))


@pytest.mark.parametrize("opt", ["{pel:1}", "{pel:2}", "{pel:4}", "{pel:2, scale:{down:2}}"])
def test_oracle16_equals_oracle8_on_8bit_samples(opt):
    # Super with bilinear planes and the 6-tap reduce has no negative taps: on samples <= 255
    # nothing reaches a clamp, so the 16-bit build must give the 8-bit build's values
    from svpflow_b200.synth import make_clip

    w, h = 96, 64
    so = orc.super_opts(w, h, opt)
    c8 = make_clip(w, h, 1, seed=11)[0]
    s8 = orc.build_super(so, c8)
    s16 = orc.build_super16(so, c8.astype(np.uint16))
    assert np.array_equal(s16, s8.astype(np.uint16))


def test_oracle16_bilinear_planes_interior():
    # fill_bilinear_pel2 away from the plane edges: h = avg(x, x+1), v = avg(y, y+1),
    # hv = avg((y, x), (y+1, x+1)), rounding up
    w, h = 64, 48
    so = orc.super_opts(w, h, "{pel:2}")
    src = clip10(w, h, 1, seed=9)[0]
    sup = orc.build_super16(so, src)
    L = src[: w * h].reshape(h, w).astype(np.int64)
    planes = sup[: 4 * h * w].reshape(4, h, w).astype(np.int64)
    avg = lambda a, b: (a + b + 1) >> 1
    assert np.array_equal(planes[1][:, : w - 1], avg(L[:, : w - 1], L[:, 1:]))
    assert np.array_equal(planes[2][1: h - 1], avg(L[1: h - 1], L[2:]))
    assert np.array_equal(planes[3][1: h - 1, : w - 1], avg(L[1: h - 1, : w - 1], L[2:, 1:]))


def test_oracle16_clamps_at_1023():
    # a saturated frame stays saturated through the 6-tap reduce and the bicubic planes
    w, h = 64, 48
    so = orc.super_opts(w, h, "{pel:2, gpu:0}")
    src = np.full(w * h * 3 // 2, 1023, dtype=np.uint16)
    sup = orc.build_super16(so, src)
    assert sup.max() == 1023


def test_bits_handles_host_side():
    sv = _sv()
    s8 = sv.Super(320, 240, "{pel:2}")
    s10 = sv.Super(320, 240, "{pel:2}", bits=10)
    assert s8.bits == 8 and s10.bits == 10
    assert s10.source_len() == 2 * s8.source_len()
    assert s10.output_len() == 2 * s8.output_len()
    assert s10.sdata == s8.sdata and s10.super_height == s8.super_height
    a8 = sv.Analyse(s8.sdata, "{}", 320, 240)
    a10 = sv.Analyse(s10.sdata, "{}", 320, 240, bits=10)
    assert a10.payload_len() == a8.payload_len() and a10.vector_header() == a8.vector_header()
    with pytest.raises(ValueError, match="bits"):
        sv.Super(320, 240, "{pel:2}", bits=12)
    with pytest.raises(ValueError, match="bits"):
        sv.Analyse(s8.sdata, "{}", 320, 240, bits=9)


# ---------------------------------------------------------------- GPU

SUPER16 = [
    (320, 240, "{pel:1}"),
    (320, 240, "{pel:2}"),
    (320, 240, "{pel:4}"),
    (320, 240, "{pel:2, gpu:0}"),     # bicubic sub-pixel planes
    (66, 38, "{pel:2}"),
    (1280, 720, "{pel:2}"),
]


@pytest.mark.gpu
@pytest.mark.parametrize("w,h,opt", SUPER16)
def test_super16_matches_oracle(w, h, opt):
    sv = _sv()
    clip = clip10(w, h, 2, seed=w + h)
    sb = sv.Super(w, h, opt, bits=10)
    so = orc.super_opts(w, h, opt)
    got = sb.build_many(clip)
    assert got.dtype == np.uint16
    want = orc.build_super_many16(so, clip)
    for i in range(clip.shape[0]):
        if not np.array_equal(got[i], want[i]):
            bad = np.nonzero(got[i] != want[i])[0]
            pytest.fail(f"frame {i}: {len(bad)} samples differ, first at {bad[0]} (row {bad[0] // w})")


ANALYSE16 = [
    (320, 180, "{pel:2}", "{block:{w:16,overlap:3},main:{search:{type:3,distance:16,satd:true}}}", 3),
    (256, 144, "{pel:2}", "{}", 2),
    (256, 144, "{pel:1}", "{block:{w:8,overlap:3},main:{search:{type:4,distance:8,satd:true,coarse:{type:2}}}}", 2),
    (256, 144, "{pel:4}", "{block:{w:8,overlap:3},main:{search:{type:4,distance:4,satd:true,coarse:{type:2}}}}", 2),
    (256, 160, "{pel:2}", "{block:{w:32,overlap:1},main:{search:{type:3,distance:8}}}", 2),
    (192, 128, "{pel:2}", "{block:{w:4,overlap:0},main:{search:{type:2,distance:4}}}", 2),
    (192, 128, "{pel:2}", "{vectors:1,block:{w:16,overlap:2},main:{search:{type:3,distance:6}}}", 2),
    (192, 128, "{pel:2}", "{main:{search:{coarse:{distance:-6,bad:{range:5}}}}}", 2),
    (192, 128, "{pel:2}", "{refine:[{thsad:200,search:{type:2,distance:3,satd:true}}]}", 2),
    (256, 144, "{pel:2, gpu:0}", "{block:{w:16,h:8,overlap:2},main:{search:{type:3,distance:6,satd:true}}}", 2),
]


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(len(ANALYSE16)))
def test_analyse16_matches_oracle(case):
    sv = _sv()
    w, h, sopt, aopt, n = ANALYSE16[case]
    clip = clip10(w, h, n, seed=300 + case, motion=6, objects=3, object_motion=10)
    sb = sv.Super(w, h, sopt, bits=10)
    an = sv.Analyse(sb.sdata, aopt, w, h, bits=10)
    so = orc.super_opts(w, h, sopt)
    ao = orc.analyse_opts(orc.sdata(so), aopt, None, w, h)
    supers = orc.build_super_many16(so, clip)
    want = orc.analyse_clip16(ao, so, supers, 0, n)
    got = an.analyse_clip(sb, clip)
    for i in range(n):
        assert got[i].tobytes() == want[i].tobytes(), f"output frame {i}: " + first_difference(got[i], want[i])


@pytest.mark.gpu
def test_analyse16_single_pair_and_device_clip():
    import torch

    sv = _sv()
    w, h, n = 320, 240, 4
    sopt, aopt = "{pel:2}", "{block:{w:16,overlap:2},main:{search:{type:3,distance:8,satd:true}}}"
    clip = clip10(w, h, n, seed=77)
    sb = sv.Super(w, h, sopt, bits=10)
    an = sv.Analyse(sb.sdata, aopt, w, h, bits=10)
    so = orc.super_opts(w, h, sopt)
    ao = orc.analyse_opts(orc.sdata(so), aopt, None, w, h)
    supers = orc.build_super_many16(so, clip)
    want = orc.analyse_clip16(ao, so, supers, 0, n)
    # host super frames, one pair
    assert an.analyse(supers[0], supers[1]) == want[0].tobytes()
    # device-resident clip through the allocation-free-of-its-own entry points
    dev = torch.device("cuda:0")
    frames_d = torch.from_numpy(clip.view(np.uint8).copy()).to(dev)
    supers_d = torch.empty((n, sb.output_len()), dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    sb.build_device(frames_d.data_ptr(), supers_d.data_ptr(), n, stream)
    pay_d = torch.empty((n, an.payload_len()), dtype=torch.uint8, device=dev)
    scr_d = torch.empty(an.scratch_bytes(n), dtype=torch.uint8, device=dev)
    an.analyse_clip_device(supers_d.data_ptr(), n, 0, n, pay_d.data_ptr(), scr_d.data_ptr(), stream)
    sv.Analyser.device_status(scr_d.data_ptr(), stream)
    assert np.array_equal(supers_d.cpu().numpy().view(np.uint16), supers)
    assert np.array_equal(pay_d.cpu().numpy(), want)


@pytest.mark.gpu
def test_batch_and_server_reject_16bit():
    sv = _sv()
    sb = sv.Super(64, 48, "{pel:2}", bits=10)
    an = sv.Analyse(sb.sdata, "{}", 64, 48, bits=10)
    with pytest.raises(sv.SvpfError, match="8-bit"):
        sv.Batch([(sb, an, 2)])
    srv = sv.Server(1 << 30, max_active=1, chunk_pairs=4)
    try:
        with pytest.raises(sv.SvpfError, match="8-bit"):
            srv.submit(sb, an, clip10(64, 48, 2, seed=1))
    finally:
        srv.close()


@pytest.mark.gpu
def test_device_entries_refuse_misaligned_buffers():
    # payload words, 8-byte scratch fields and 16-bit samples would fault at unaligned addresses:
    # each entry point refuses them before launching (the buffers are real and large enough)
    import torch

    sv = _sv()
    w, h, n = 64, 48, 2
    sb8 = sv.Super(w, h, "{pel:2}")
    an8 = sv.Analyse(sb8.sdata, "{}", w, h)
    sb10 = sv.Super(w, h, "{pel:2}", bits=10)
    an10 = sv.Analyse(sb10.sdata, "{}", w, h, bits=10)
    big = lambda k: torch.zeros(k + 64, dtype=torch.uint8, device="cuda")
    sup8, sup10 = big(n * sb8.output_len()), big(n * sb10.output_len())
    frames10 = big(n * sb10.source_len())
    pay = big(n * max(an8.payload_len(), an10.payload_len()))
    scr = big(max(an8.scratch_bytes(n), an10.scratch_bytes(n)))
    sv.reset_kernel_launches()
    with pytest.raises(ValueError, match="payloads"):
        an8.analyse_clip_device(sup8.data_ptr(), n, 0, 1, pay.data_ptr() + 2, scr.data_ptr())
    with pytest.raises(ValueError, match="scratch"):
        an8.analyse_clip_device(sup8.data_ptr(), n, 0, 1, pay.data_ptr(), scr.data_ptr() + 8)
    with pytest.raises(ValueError, match="payloads"):
        an8.analyse_pairs_device([sup8.data_ptr()], [sup8.data_ptr() + sb8.output_len()], pay.data_ptr() + 1,
                                 scr.data_ptr())
    with pytest.raises(ValueError, match="2-byte"):
        sb10.build_device(frames10.data_ptr() + 1, sup10.data_ptr(), n)
    with pytest.raises(ValueError, match="2-byte"):
        an10.analyse_clip_device(sup10.data_ptr() + 1, n, 0, 1, pay.data_ptr(), scr.data_ptr())
    assert sv.kernel_launches() == 0
