"""The batched and served forms (GPU): every payload equals the oracle's (the CPU
restatement of the reference, on the same frames and options) and the plain per-clip
path's, for every launch shape, alone and in a mix of clips of uneven size, length and
options; served clips overlap on the device. Tolerance: zero (integer work)."""
import os

import numpy as np
import pytest

from oracle import oracle as orc

pytestmark = pytest.mark.gpu

# (w, h, frames, seed, super opt, analyse opt)
MIX = [
    (192, 128, 5, 11, "{pel:2}", "{block:{w:16,overlap:3},main:{search:{type:3,distance:8,satd:true}}}"),
    (128, 96, 3, 12, "{pel:2}", "{block:{w:8,overlap:2},main:{search:{type:3,distance:6,satd:true}}}"),
    (160, 96, 4, 13, "{pel:1}", "{vectors:1,block:{w:16,overlap:0},main:{search:{type:2,distance:2}}}"),
    (256, 144, 2, 14, "{pel:4}", "{block:{w:8,overlap:3},main:{search:{type:4,distance:3,satd:true,coarse:{type:2}}}}"),
    (96, 64, 6, 15, "{pel:2}", "{vectors:2,delta:2,block:{w:8,overlap:1},main:{search:{type:2,distance:4}}}"),
]


def _clips(mix=MIX):
    import svpflow_b200 as sv
    from svpflow_b200.synth import make_clip

    out = []
    for w, h, n, seed, sopt, aopt in mix:
        sb = sv.Super(w, h, sopt)
        an = sv.Analyse(sb.sdata, aopt, w, h)
        clip = make_clip(w, h, n, seed=seed, motion=6, objects=2, object_motion=9)
        out.append((sb, an, clip))
    return out


def _plain(clips):
    return [an.analyse_clip(sb, clip) for sb, an, clip in clips]


def _oracle(clips, mix=MIX):
    """Every output frame of every clip from the oracle (frame n pairs with min(n + delta, last))."""
    out = []
    for (sb, an, clip), (w, h, n, _, sopt, aopt) in zip(clips, mix):
        so = orc.super_opts(w, h, sopt)
        ao = orc.analyse_opts(orc.sdata(so), aopt, None, w, h)
        supers = orc.build_super_many(so, clip, os.cpu_count() or 1)
        out.append(orc.analyse_clip(ao, so, supers, 0, n, os.cpu_count() or 1))
    return out


def _expect(clips, mix=MIX):
    """The oracle's payloads, after checking that the plain per-clip path gives the same."""
    want = _oracle(clips, mix)
    for i, (g, w_) in enumerate(zip(_plain(clips), want)):
        assert np.array_equal(g, w_), f"plain path: clip {i} differs from the oracle"
    return want


class _Dev:
    """A raw device byte range as a torch tensor (CUDA array interface; no copy)."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "|u1", "data": (ptr, False), "version": 3}


def _dev(ptr, n):
    import torch

    return torch.as_tensor(_Dev(ptr, n), device="cuda")


def test_batch_matches_plain_for_every_shape():
    import svpflow_b200 as sv

    clips = _clips()
    want = _expect(clips)
    b = sv.Batch([(sb, an, clip.shape[0]) for sb, an, clip in clips])
    assert b.pairs == sum(c[2].shape[0] for c in clips)
    for v in range(len(sv.Batch.variants())):
        for t in (2, 4, 8):
            b.set_shape(v, t)
            got = b.run([c[2] for c in clips])
            for i, (g, w_) in enumerate(zip(got, want)):
                assert np.array_equal(g, w_), f"variant {v} tiles/lane {t}: clip {i} differs"
    b.close()


def test_batch_device_replay_and_autotune():
    import torch

    import svpflow_b200 as sv

    clips = _clips(MIX[:3])
    want = _expect(clips, MIX[:3])
    b = sv.Batch([(sb, an, clip.shape[0]) for sb, an, clip in clips])
    for i, (_, _, clip) in enumerate(clips):  # fill the batch's frame buffers on the device
        ptr = b.frames_device(i)
        assert ptr
        _dev(ptr, clip.size).copy_(torch.from_numpy(clip.reshape(-1)))
    torch.cuda.synchronize()
    for _ in range(2):  # graph replays
        b.launch()
        b.status()
        for i, (_, an, clip) in enumerate(clips):
            n, L = clip.shape[0], an.payload_len()
            got = _dev(b.payloads_device(i), n * L).cpu().numpy().reshape(n, L)
            assert np.array_equal(got, want[i])
    r = b.autotune()
    assert 0 <= r["variant"] < len(sv.Batch.variants()) and r["tiles_per_lane"] in (2, 4, 8)
    assert r["trial_pairs_per_s"] > 0
    got = b.run([c[2] for c in clips])
    assert all(np.array_equal(g, w_) for g, w_ in zip(got, want))
    b.close()


def test_server_results_equal_alone_and_in_the_mix():
    import time

    import svpflow_b200 as sv

    clips = _clips()
    want = _expect(clips)
    # a budget below two of the largest clips, so admission has to wait for memory
    chunk = 2
    need = [c[2].nbytes + (c[0].output_len() + c[1].payload_len()) * c[2].shape[0] +
            c[1].scratch_bytes(min(chunk, c[2].shape[0])) + 2048 for c in clips]
    budget = int(1.6 * max(need))
    srv = sv.Server(budget, max_active=3, chunk_pairs=chunk)
    try:
        ids = []
        for k, (sb, an, clip) in enumerate(clips):
            ids.append(srv.submit(sb, an, clip))
            time.sleep(0.01 * (k % 2))
        for k, rid in enumerate(ids):
            pay, done, (arr, adm, fin) = srv.wait(rid)
            assert np.array_equal(pay, want[k]), f"clip {k} differs in the mix"
            assert arr <= adm <= fin and (done >= arr).all() and (done <= fin).all()
        st = srv.stats()
        assert st["completed"] == len(clips) and 1 <= st["peak_active"] <= 3
        assert st["peak_device_bytes"] <= budget and st["kernel_launches"] > 0
        # the same clip alone on the same server
        sb, an, clip = clips[0]
        pay, _, _ = srv.wait(srv.submit(sb, an, clip))
        assert np.array_equal(pay, want[0])
    finally:
        srv.close()


def test_server_rejects_a_clip_over_budget():
    import svpflow_b200 as sv

    (sb, an, clip), = _clips(MIX[:1])
    srv = sv.Server(1 << 20, max_active=2, chunk_pairs=4)
    try:
        with pytest.raises(ValueError, match="more device memory than the server's budget"):
            srv.submit(sb, an, clip)
    finally:
        srv.close()


def test_served_clips_overlap_on_the_device():
    """Continuous batching: clips admitted together run concurrently on the GPU. Four copies of a
    small clip, served with four slots, finish in clearly less than four times the span of one copy
    served alone (one after another they would take at least four times as long: a clip's span is
    its own device work plus its copies), and every copy's payloads equal the oracle's. The margin
    allows for the level-0 kernel, which spreads even one small clip's warps over every SM."""
    import svpflow_b200 as sv

    mix = [(640, 360, 9, 21, "{pel:2}", "{block:{w:16,overlap:3},main:{search:{type:3,distance:8,satd:true}}}")]
    (sb, an, clip), = _clips(mix)
    want = _expect([(sb, an, clip)], mix)[0]
    srv = sv.Server(8 << 30, max_active=4, chunk_pairs=16)
    try:
        srv.wait(srv.submit(sb, an, clip))  # warm-up (module load, pools)
        spans_alone = []
        for _ in range(3):
            pay, _, (arr, _, fin) = srv.wait(srv.submit(sb, an, clip))
            spans_alone.append(fin - arr)
            assert np.array_equal(pay, want)
        alone = min(spans_alone)
        ids = [srv.submit(sb, an, clip) for _ in range(4)]
        res = [srv.wait(r) for r in ids]
        t0 = min(r[2][0] for r in res)
        t1 = max(r[2][2] for r in res)
        for pay, _, _ in res:
            assert np.array_equal(pay, want)
        assert srv.stats()["peak_active"] >= 2
        assert (t1 - t0) < 3.2 * alone, f"four clips took {(t1 - t0) / 1e6:.1f} ms, one alone {alone / 1e6:.1f} ms"
    finally:
        srv.close()


def test_server_cancels_a_request_before_admission():
    """svpf_server_cancel withdraws a queued request (its wait reports SVPF_ECANCELED and it never
    runs); admitted, finished and unknown requests cannot be cancelled; the requests around the
    cancelled one complete with the oracle's payloads."""
    import svpflow_b200 as sv

    mix = [(1280, 720, 12, 31, "{pel:2}", "{block:{w:16,overlap:3},main:{search:{type:3,distance:16,satd:true}}}"),
           (192, 128, 3, 32, "{pel:2}", "{block:{w:8,overlap:2},main:{search:{type:3,distance:6,satd:true}}}"),
           (160, 96, 4, 33, "{pel:1}", "{vectors:1,block:{w:16,overlap:0},main:{search:{type:2,distance:2}}}")]
    clips = _clips(mix)
    want = _oracle(clips, mix)
    import time

    srv = sv.Server(8 << 30, max_active=1, chunk_pairs=4)
    try:
        ids = [srv.submit(*clips[0])]
        t0 = time.time()
        while srv.stats()["admitted"] < 1 and time.time() - t0 < 10:  # the scheduler thread takes it up
            time.sleep(0.001)
        ids += [srv.submit(sb, an, clip) for sb, an, clip in clips[1:]]  # one slot: these wait for the 1st
        srv.cancel(ids[1])
        with pytest.raises(ValueError, match="admitted|finished"):
            srv.cancel(ids[0])
        with pytest.raises(ValueError, match="unknown request"):
            srv.cancel(10 ** 9)
        with pytest.raises(sv.SvpfError) as e:
            srv.wait(ids[1])
        assert e.value.code == sv.SVPF_ECANCELED
        for k in (0, 2):
            pay, _, _ = srv.wait(ids[k])
            assert np.array_equal(pay, want[k]), f"clip {k} differs from the oracle"
        st = srv.stats()
        assert st["admitted"] == 2 and st["completed"] == 2
    finally:
        srv.close()
