"""The allocation-free Analyse entry point, svpf_clip_analyse_device_noalloc.

It exists for callers that may not allocate device memory (a frame server's per-frame
callback, or a host that forbids allocations after start-up); its scratch is a fixed
array inside the library. Called through the C ABI, twice in a row, after a call on
another clip with other options has left its own data in the array, it must give the
same payloads as svpf_clip_analyse_device with caller-provided scratch: the work is
integer, so the tolerance is zero (byte equality). Requests beyond the fixed array are
rejected with SVPF_EINVAL before anything is launched.

This file is collected last on purpose (a failure here leaves every other test run).
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SVPF_EINVAL = -1


def _noalloc(lib):
    f = lib.svpf_clip_analyse_device_noalloc
    f.restype = ctypes.c_int32
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                  ctypes.c_void_p, ctypes.c_void_p]
    return f


def _setup(w, h, nframes, sopt, aopt, seed):
    import torch

    import svpflow_b200 as sv
    from svpflow_b200.synth import make_clip

    clip = make_clip(w, h, nframes, seed=seed, motion=6, objects=3, object_motion=10)
    sb = sv.Super(w, h, sopt)
    an = sv.Analyse(sb.sdata, aopt, w, h)
    dev = torch.device("cuda", 0)
    frames = torch.from_numpy(clip).to(dev)
    supers = torch.empty((nframes, sb.output_len()), dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    sb.build_device(frames.data_ptr(), supers.data_ptr(), nframes, stream)
    return sv, an, supers, stream


def _with_scratch(sv, an, supers, n, stream):
    """The payloads of the existing entry point, svpf_clip_analyse_device, with caller scratch."""
    import torch

    dev = supers.device
    want = torch.empty((n, an.payload_len()), dtype=torch.uint8, device=dev)
    scratch = torch.empty(an.scratch_bytes(n), dtype=torch.uint8, device=dev)
    an.analyse_clip_device(supers.data_ptr(), n, 0, n, want.data_ptr(), scratch.data_ptr(), stream)
    sv.Analyser.device_status(scratch.data_ptr(), stream)
    return want


def test_noalloc_matches_clip_analyse_device_twice():
    import torch

    # First a different clip with other options (block 8, exhaustive search, one direction,
    # another grid and payload length), so the shared array holds another call's leftovers when
    # the checked calls run: they must not read anything they did not write themselves.
    m = 4
    sv, an_o, supers_o, stream = _setup(
        256, 144, m, "{pel:1}", "{vectors:1,block:{w:8,overlap:1},main:{search:{type:4,distance:4}}}", seed=3)
    f = _noalloc(sv.lib())
    other = torch.full((m, an_o.payload_len()), 0x5A, dtype=torch.uint8, device=supers_o.device)
    rc = f(an_o.handle, supers_o.data_ptr(), m, 0, m, other.data_ptr(), stream)
    assert rc == 0, sv.lib().svpf_last_error().decode()
    want_o = _with_scratch(sv, an_o, supers_o, m, stream)
    assert np.array_equal(other.cpu().numpy(), want_o.cpu().numpy()), "the first clip's payloads differ"

    n = 5
    sv, an, supers, stream = _setup(
        320, 180, n, "{pel:2}", "{block:{w:16,overlap:3},main:{search:{type:3,distance:16,satd:true}}}", seed=11)
    pl = an.payload_len()
    dev = supers.device
    want = _with_scratch(sv, an, supers, n, stream)
    for call in range(2):
        got = torch.full((n, pl), 0xA5, dtype=torch.uint8, device=dev)
        rc = f(an.handle, supers.data_ptr(), n, 0, n, got.data_ptr(), stream)
        assert rc == 0, sv.lib().svpf_last_error().decode()
        torch.cuda.synchronize()
        assert np.array_equal(got.cpu().numpy(), want.cpu().numpy()), f"call {call}: payloads differ"


def test_noalloc_rejects_requests_above_its_scratch():
    import torch

    # 40 pairs of 320x180 with 4x4 blocks need about 37 MB of scratch, above the 32 MiB
    # array. The buffers are real and sized for the request, so nothing is out of range
    # even though the call must refuse before launching anything.
    n = 40
    sv, an, supers, stream = _setup(320, 180, n + 1, "{pel:2}", "{block:{w:4,overlap:0},main:{search:{type:2,distance:2}}}",
                                    seed=5)
    assert an.scratch_bytes(n) > 32 << 20
    out = torch.empty((n, an.payload_len()), dtype=torch.uint8, device=supers.device)
    f = _noalloc(sv.lib())
    sv.reset_kernel_launches()
    rc = f(an.handle, supers.data_ptr(), n + 1, 0, n, out.data_ptr(), stream)
    assert rc == SVPF_EINVAL
    assert "static scratch" in sv.lib().svpf_last_error().decode()
    assert sv.kernel_launches() == 0


def test_noalloc_rejects_misaligned_payloads():
    import torch

    # payload words are written 4 bytes at a time: an unaligned buffer is refused before any launch
    n = 2
    sv, an, supers, stream = _setup(64, 48, n + 1, "{pel:2}", "{}", seed=6)
    out = torch.empty(n * an.payload_len() + 16, dtype=torch.uint8, device=supers.device)
    f = _noalloc(sv.lib())
    sv.reset_kernel_launches()
    rc = f(an.handle, supers.data_ptr(), n + 1, 0, n, out.data_ptr() + 2, stream)
    assert rc == SVPF_EINVAL
    assert "aligned" in sv.lib().svpf_last_error().decode()
    assert sv.kernel_launches() == 0
