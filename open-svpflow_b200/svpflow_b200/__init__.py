"""svpflow_b200 -- host-side mirror of open-svpflow's motion-analysis interface.

Python face of libsvpflow_b200.so (the C ABI in include/svpflow_b200.h). Names and
argument meanings follow the reference:

  SuperBuilder / SuperFrame / Analyser   crates/svpflow1/src/portable.rs:8-251
  Super(width, height, opt)              the `svp1.Super` filter, super_filter.rs:9-105
  Analyse(sdata, opt, width, height)     the `svp1.Analyse` filter, analyse_filter.rs:29-171

Errors raise ValueError with the reference's message text. Everything computes on the
GPU; without a usable CUDA device or without the compiled library the calls fail
loudly -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence

import numpy as np

__all__ = ["SuperBuilder", "SuperFrame", "Analyser", "Super", "Analyse", "Batch", "Server", "lib", "LIB_PATH",
           "SvpfError", "REFERENCE_VERSION"]

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(HERE), "lib", "libsvpflow_b200.so")
REFERENCE_VERSION = 1_174_405_393  # svpGetVersion, crates/svpflow1/src/abi.rs:3

SVPF_OK, SVPF_EINVAL, SVPF_ECUDA, SVPF_EPANIC, SVPF_EUNSUP, SVPF_ECANCELED = 0, -1, -2, -3, -4, -5


class SvpfError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


_lib = None
_VP = ctypes.c_void_p


class RenderConfig(ctypes.Structure):
    """svpf_render_config: renderer.rs CpuConfig as SmoothFps fills it."""
    _fields_ = [(f, ctypes.c_int32) for f in ("width", "height", "block_w", "block_h", "origin_x", "origin_y",
                                               "grid_w", "grid_h", "source_step")]


class SceneLimits(ctypes.Structure):
    """svpf_scene_limits: SmoothFps's scene limits."""
    _fields_ = [(f, ctypes.c_int32) for f in ("blocks_pct", "zero", "m1", "m2", "scene")]


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} is not built: run `python __graft_entry__.py` (build()) first")
        L = ctypes.CDLL(LIB_PATH)
        P, I32, I64, SZ = ctypes.POINTER, ctypes.c_int32, ctypes.c_int64, ctypes.c_size_t
        sig = {
            "svpf_last_error": (ctypes.c_char_p, []),
            "svpf_reference_version": (I64, []),
            "svpf_super_create": (I32, [I32, I32, ctypes.c_char_p, SZ, P(_VP)]),
            "svpf_super_create_portable": (I32, [I32, I32, I32, P(_VP)]),
            "svpf_super_create_bits": (I32, [I32, I32, ctypes.c_char_p, SZ, I32, P(_VP)]),
            "svpf_super_bits": (I32, [_VP]),
            "svpf_analyser_create_bits": (I32, [I64, ctypes.c_char_p, SZ, I32, I32, I32, P(_VP)]),
            "svpf_super_destroy": (None, [_VP]),
            "svpf_super_sdata": (I64, [_VP]),
            "svpf_super_height": (I32, [_VP]),
            "svpf_super_levels": (I32, [_VP]),
            "svpf_super_pel": (I32, [_VP]),
            "svpf_super_source_len": (SZ, [_VP]),
            "svpf_super_output_len": (SZ, [_VP]),
            "svpf_super_build": (I32, [_VP, _VP, _VP, I32]),
            "svpf_super_build_device": (I32, [_VP, _VP, I64, I64, _VP, I32, _VP]),
            "svpf_analyser_create": (I32, [I64, ctypes.c_char_p, SZ, I32, I32, P(_VP)]),
            "svpf_analyser_create_portable": (I32, [_VP, I32, I32, I32, I32, P(_VP)]),
            "svpf_analyser_destroy": (None, [_VP]),
            "svpf_analyser_vdata": (P(I32), [_VP]),
            "svpf_analyser_payload_len": (SZ, [_VP]),
            "svpf_analyser_delta": (I32, [_VP]),
            "svpf_analyser_scratch_bytes": (SZ, [_VP, I32]),
            "svpf_analyse": (I32, [_VP, _VP, _VP, _VP]),
            "svpf_analyse_pairs_device": (I32, [_VP, P(_VP), P(_VP), I32, _VP, _VP, _VP]),
            "svpf_clip_analyse_device": (I32, [_VP, _VP, I32, I32, I32, _VP, _VP, _VP]),
            "svpf_device_status": (I32, [_VP, _VP]),
            "svpf_analyser_set_lookahead": (I32, [_VP, I32]),
            "svpf_device_lookahead_stats": (I32, [_VP, _VP, P(I64)]),
            "svpf_clip_analyse": (I32, [_VP, _VP, _VP, I32, I32, I32, _VP]),
            "svpf_kernel_launches": (I64, []),
            "svpf_kernel_launches_reset": (None, []),
            "svpf_batch_create": (I32, [I32, P(_VP), P(_VP), P(I32), P(_VP)]),
            "svpf_batch_destroy": (None, [_VP]),
            "svpf_batch_clips": (I32, [_VP]),
            "svpf_batch_pairs": (I64, [_VP]),
            "svpf_batch_device_bytes": (SZ, [_VP]),
            "svpf_batch_frames_device": (_VP, [_VP, I32]),
            "svpf_batch_payloads_device": (_VP, [_VP, I32]),
            "svpf_batch_run": (I32, [_VP, P(_VP), P(_VP)]),
            "svpf_batch_launch": (I32, [_VP, _VP]),
            "svpf_batch_status": (I32, [_VP, _VP]),
            "svpf_batch_set_shape": (I32, [_VP, I32, I32]),
            "svpf_batch_shape": (ctypes.c_char_p, [_VP, P(I32), P(I32), P(I32)]),
            "svpf_batch_autotune": (I32, [_VP, P(I32), P(I32), P(ctypes.c_double)]),
            "svpf_batch_graph_launches": (I32, [_VP]),
            "svpf_analyse_variant_count": (I32, []),
            "svpf_analyse_variant_name": (ctypes.c_char_p, [I32]),
            "svpf_server_create": (I32, [SZ, I32, I32, P(_VP)]),
            "svpf_server_destroy": (None, [_VP]),
            "svpf_server_submit": (I32, [_VP, _VP, _VP, _VP, I32, _VP, _VP, P(I64)]),
            "svpf_server_wait": (I32, [_VP, I64, P(I64)]),
            "svpf_server_cancel": (I32, [_VP, I64]),
            "svpf_server_now_ns": (I64, [_VP]),
            "svpf_server_stats": (None, [_VP, P(I64), P(I64), P(I64), P(I32), P(I64)]),
            "svpf_vector_grid": (I32, [P(I32), P(I32), P(I32)]),
            "svpf_vector_planes_device": (I32, [P(I32), _VP, SZ, I32, I32, I32, I32, _VP, _VP, _VP]),
            "svpf_scene_class_device": (I32, [P(I32), _VP, SZ, I32, ctypes.c_double, P(SceneLimits), _VP, _VP,
                                              _VP]),
            "svpf_render_masks_scratch": (I64, [P(I32), I32]),
            "svpf_render_masks_device": (I32, [P(I32), _VP, SZ, I32, I32, I32, ctypes.c_double, ctypes.c_double,
                                               _VP, _VP, _VP, _VP]),
            "svpf_render_warp_device": (I32, [P(RenderConfig), I32, I32, I32, P(_VP), P(I64), P(I64), I32, _VP, _VP,
                                              _VP, P(_VP), P(I64), _VP]),
            "svpf_render_blend_device": (I32, [P(RenderConfig), I32, I32, I32, I32, P(_VP), P(I64), P(I64), P(_VP),
                                               P(I64), P(I64), I32, _VP, _VP, _VP, _VP, _VP, _VP, P(_VP), P(I64),
                                               _VP]),
            "svpf_render_masked_device": (I32, [P(RenderConfig), I32, ctypes.c_double, I32, I32, P(_VP), P(I64),
                                                P(I64), P(_VP), P(I64), P(I64), I32, _VP, _VP, _VP, _VP, _VP, _VP,
                                                _VP, P(_VP), P(I64), _VP]),
            "svpf_render_mode23_device": (I32, [P(RenderConfig), I32, I32, P(_VP), P(I64), P(I64), P(_VP), P(I64),
                                                P(I64), I32, P(_VP), P(_VP), _VP, _VP, _VP, P(_VP), P(I64), _VP]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(rc: int):
    if rc != SVPF_OK:
        msg = lib().svpf_last_error().decode(errors="replace")
        if rc == SVPF_EINVAL:
            raise ValueError(msg)
        raise SvpfError(rc, msg)


def _buf(a) -> np.ndarray:
    """Bytes of a buffer: uint8 data as is, uint16 samples (the 10-bit extension) viewed as bytes."""
    if isinstance(a, (bytes, bytearray, memoryview)):
        return np.frombuffer(a, dtype=np.uint8)
    if isinstance(a, np.ndarray) and a.dtype == np.uint16:
        return np.ascontiguousarray(a).reshape(-1).view(np.uint8)
    return np.ascontiguousarray(a, dtype=np.uint8)


def _sample_type(bits: int):
    return np.uint16 if bits > 8 else np.uint8


class SuperFrame:
    """A super frame in the portable layout (portable.rs:151-186)."""

    def __init__(self, builder: "SuperBuilder", data: np.ndarray):
        self.builder = builder
        self.data = data

    def bytes(self) -> bytes:
        return self.data.tobytes()

    def __len__(self) -> int:
        return int(self.data.size)


class SuperBuilder:
    """SuperBuilder::new(width, height, pel) (portable.rs:29-62); Super(...) for the filter form."""

    def __init__(self, width: int, height: int, pel: int = 2, *, _handle=None):
        h = _VP()
        if _handle is None:
            _check(lib().svpf_super_create_portable(width, height, pel, ctypes.byref(h)))
        else:
            h = _handle
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.svpf_super_destroy(self._h)
            self._h = None

    @property
    def handle(self):
        return self._h

    @property
    def levels(self) -> int:
        return lib().svpf_super_levels(self._h)

    @property
    def pel(self) -> int:
        return lib().svpf_super_pel(self._h)

    @property
    def sdata(self) -> int:
        """The `data` int the Super filter publishes (SuperOpts::pack_data)."""
        return lib().svpf_super_sdata(self._h)

    @property
    def super_height(self) -> int:
        return lib().svpf_super_height(self._h)

    @property
    def bits(self) -> int:
        """Sample depth: 8 (the reference's), or 10 (uint16 samples; this project's extension)."""
        return lib().svpf_super_bits(self._h)

    @property
    def sample_type(self):
        return _sample_type(self.bits)

    def source_len(self) -> int:
        """Bytes of one packed I420 source frame."""
        return lib().svpf_super_source_len(self._h)

    def output_len(self) -> int:
        """Bytes of one super frame."""
        return lib().svpf_super_output_len(self._h)

    def build(self, source) -> SuperFrame:
        """SuperBuilder::build: one packed I420 frame -> its super frame."""
        dt = self.sample_type
        src = np.ascontiguousarray(source, dtype=dt) if dt is np.uint16 else _buf(source)
        if src.nbytes != self.source_len():
            raise ValueError("invalid source buffer length")
        out = np.empty(self.output_len() // np.dtype(dt).itemsize, dtype=dt)
        _check(lib().svpf_super_build(self._h, src.ctypes.data, out.ctypes.data, 1))
        return SuperFrame(self, out)

    def build_many(self, frames: np.ndarray) -> np.ndarray:
        dt = self.sample_type
        frames = np.ascontiguousarray(frames, dtype=dt)
        n = frames.shape[0]
        if frames.nbytes != n * self.source_len():
            raise ValueError("invalid source buffer length")
        out = np.empty((n, self.output_len() // np.dtype(dt).itemsize), dtype=dt)
        _check(lib().svpf_super_build(self._h, frames.ctypes.data, out.ctypes.data, n))
        return out

    def build_device(self, src_ptr: int, dst_ptr: int, nframes: int, stream: int = 0,
                     src_y_stride: int = 0, src_c_stride: int = 0):
        """Device buffers (e.g. torch tensors' data_ptr()) on `stream`; no allocation."""
        _check(lib().svpf_super_build_device(self._h, src_ptr, src_y_stride, src_c_stride, dst_ptr, nframes, stream))


def Super(width: int, height: int, opt: Optional[str] = None, bits: int = 8) -> SuperBuilder:
    """The `svp1.Super(clip, opt)` filter's configuration for a clip of this size. bits=10 is this
    project's 10-bit extension (uint16 samples); the reference is 8-bit only."""
    h = _VP()
    b = opt.encode() if opt is not None else None
    if bits == 8:
        _check(lib().svpf_super_create(width, height, b, len(b) if b else 0, ctypes.byref(h)))
    else:
        _check(lib().svpf_super_create_bits(width, height, b, len(b) if b else 0, bits, ctypes.byref(h)))
    return SuperBuilder(0, 0, _handle=h)


class Analyser:
    """Analyser::new(super_builder, block w, block h, overlap mode, vectors) (portable.rs:188-250);
    Analyse(...) for the filter form."""

    def __init__(self, super_builder: Optional[SuperBuilder] = None, block_width: int = 16, block_height: int = 16,
                 overlap_mode: int = 2, vectors: int = 3, *, _handle=None, _bits: int = 8):
        self.bits = super_builder.bits if super_builder is not None and _handle is None else _bits
        h = _VP()
        if _handle is None:
            _check(lib().svpf_analyser_create_portable(super_builder.handle, block_width, block_height, overlap_mode,
                                                        vectors, ctypes.byref(h)))
        else:
            h = _handle
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.svpf_analyser_destroy(self._h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def vector_header(self) -> list:
        """The `vdata` header (pack_vdata_header)."""
        p = lib().svpf_analyser_vdata(self._h)
        return [p[i] for i in range(16)]

    def payload_len(self) -> int:
        return lib().svpf_analyser_payload_len(self._h)

    @property
    def delta(self) -> int:
        return lib().svpf_analyser_delta(self._h)

    def scratch_bytes(self, npairs: int) -> int:
        return lib().svpf_analyser_scratch_bytes(self._h, npairs)

    def analyse(self, current, reference) -> bytes:
        """Analyser::analyse(current, reference) -> the Analyse output frame bytes."""
        cur = _buf(current.data if isinstance(current, SuperFrame) else current)
        ref = _buf(reference.data if isinstance(reference, SuperFrame) else reference)
        out = np.empty(self.payload_len(), dtype=np.uint8)
        _check(lib().svpf_analyse(self._h, cur.ctypes.data, ref.ctypes.data, out.ctypes.data))
        return out.tobytes()

    def analyse_clip(self, super_builder: SuperBuilder, frames: np.ndarray, first: int = 0,
                     count: Optional[int] = None) -> np.ndarray:
        """Super + Analyse over a clip of packed I420 frames (host buffers) -> payload rows."""
        frames = np.ascontiguousarray(frames, dtype=_sample_type(self.bits))
        n = frames.shape[0]
        if frames.nbytes != n * super_builder.source_len():
            raise ValueError("invalid source buffer length")
        count = n - first if count is None else count
        out = np.empty((count, self.payload_len()), dtype=np.uint8)
        _check(lib().svpf_clip_analyse(self._h, super_builder.handle, frames.ctypes.data, n, first, count,
                                       out.ctypes.data))
        return out

    def analyse_clip_device(self, supers_ptr: int, nframes: int, first: int, count: int, payloads_ptr: int,
                            scratch_ptr: int, stream: int = 0):
        """Device-resident clip of super frames -> payloads; caller-owned buffers, no allocation."""
        _check(lib().svpf_clip_analyse_device(self._h, supers_ptr, nframes, first, count, payloads_ptr, scratch_ptr,
                                              stream))

    def analyse_pairs_device(self, cur_ptrs: Sequence[int], ref_ptrs: Sequence[int], payloads_ptr: int,
                             scratch_ptr: int, stream: int = 0):
        n = len(cur_ptrs)
        c = (_VP * n)(*cur_ptrs)
        r = (_VP * n)(*ref_ptrs)
        _check(lib().svpf_analyse_pairs_device(self._h, c, r, n, payloads_ptr, scratch_ptr, stream))

    def set_lookahead(self, levels):
        """Look-ahead bits: 1 level 0, 2 the coarser levels, 4 level 0 spread over the GPU in a
        launch of its own (with 1). True is the default (5), False / 0 off; results are identical
        either way."""
        _check(lib().svpf_analyser_set_lookahead(self._h, 5 if levels is True else int(levels)))

    @staticmethod
    def lookahead_stats(scratch_ptr: int, stream: int = 0) -> dict:
        """Counters of the last device launch on that scratch."""
        v = (ctypes.c_int64 * 4)()
        _check(lib().svpf_device_lookahead_stats(scratch_ptr, stream, v))
        return {"blocks": v[0], "deferred_blocks": v[1], "deferred_evaluated": v[2], "reruns": v[3]}

    @staticmethod
    def device_status(scratch_ptr: int, stream: int = 0):
        _check(lib().svpf_device_status(scratch_ptr, stream))


def Analyse(sdata: int, opt: Optional[str] = None, width: int = 0, height: int = 0, bits: int = 8) -> Analyser:
    """The `svp1.Analyse(clip, sdata, src, opt)` filter's configuration; width/height are the
    src clip's size (analyse_filter.rs:96-101). bits=10: super frames of uint16 samples."""
    h = _VP()
    b = opt.encode() if opt is not None else None
    if bits == 8:
        _check(lib().svpf_analyser_create(sdata, b, len(b) if b else 0, width, height, ctypes.byref(h)))
    else:
        _check(lib().svpf_analyser_create_bits(sdata, b, len(b) if b else 0, width, height, bits, ctypes.byref(h)))
    return Analyser(_handle=h, _bits=bits)


def kernel_launches() -> int:
    return lib().svpf_kernel_launches()


def reset_kernel_launches():
    lib().svpf_kernel_launches_reset()


class Batch:
    """Many clips analysed by one persistent launch (no counterpart in the reference).

    clips: sequence of (SuperBuilder, Analyser, nframes). Payloads equal each clip's
    Analyser.analyse_clip output byte for byte."""

    def __init__(self, clips):
        self._keep = list(clips)  # the handles must outlive the batch
        n = len(self._keep)
        sups = (_VP * n)(*[c[0].handle for c in self._keep])
        ans = (_VP * n)(*[c[1].handle for c in self._keep])
        nf = (ctypes.c_int32 * n)(*[int(c[2]) for c in self._keep])
        h = _VP()
        _check(lib().svpf_batch_create(n, sups, ans, nf, ctypes.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.svpf_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    @property
    def pairs(self) -> int:
        return lib().svpf_batch_pairs(self._h)

    @property
    def device_bytes(self) -> int:
        return lib().svpf_batch_device_bytes(self._h)

    def frames_device(self, clip: int) -> int:
        return lib().svpf_batch_frames_device(self._h, clip)

    def payloads_device(self, clip: int) -> int:
        return lib().svpf_batch_payloads_device(self._h, clip)

    def run(self, frames, payloads=None):
        """Host frames per clip in, payload arrays per clip out (allocated when not given)."""
        n = len(self._keep)
        frames = [np.ascontiguousarray(f, dtype=np.uint8) for f in frames]
        if payloads is None:
            payloads = [np.empty((c[2], c[1].payload_len()), dtype=np.uint8) for c in self._keep]
        fp = (_VP * n)(*[f.ctypes.data for f in frames])
        pp = (_VP * n)(*[p.ctypes.data for p in payloads])
        _check(lib().svpf_batch_run(self._h, fp, pp))
        return payloads

    def launch(self, stream: int = 0):
        """Replays the run on `stream` (0 = the batch's own stream)."""
        _check(lib().svpf_batch_launch(self._h, stream))

    def status(self, stream: int = 0):
        _check(lib().svpf_batch_status(self._h, stream))

    def set_shape(self, variant: int, tiles_per_lane: int):
        _check(lib().svpf_batch_set_shape(self._h, variant, tiles_per_lane))

    def shape(self) -> dict:
        v, t, g = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        name = lib().svpf_batch_shape(self._h, ctypes.byref(v), ctypes.byref(t), ctypes.byref(g)).decode()
        return {"variant": v.value, "name": name, "tiles_per_lane": t.value, "grid": g.value}

    def autotune(self) -> dict:
        v, t, r = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_double()
        _check(lib().svpf_batch_autotune(self._h, ctypes.byref(v), ctypes.byref(t), ctypes.byref(r)))
        return {"trial_pairs_per_s": r.value, **self.shape()}

    @property
    def graph_launches(self) -> int:
        return lib().svpf_batch_graph_launches(self._h)

    @staticmethod
    def variants() -> list:
        return [lib().svpf_analyse_variant_name(i).decode() for i in range(lib().svpf_analyse_variant_count())]


class Server:
    """Continuous-batching request loop (no counterpart in the reference)."""

    def __init__(self, hbm_budget_bytes: int, max_active: int = 8, chunk_pairs: int = 32):
        self._live = {}
        h = _VP()
        _check(lib().svpf_server_create(int(hbm_budget_bytes), max_active, chunk_pairs, ctypes.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.svpf_server_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def now_ns(self) -> int:
        return lib().svpf_server_now_ns(self._h)

    def submit(self, super_builder: SuperBuilder, analyser: Analyser, frames: np.ndarray, payloads: np.ndarray = None,
               pair_done_ns: np.ndarray = None) -> int:
        frames = np.ascontiguousarray(frames, dtype=np.uint8)
        n = frames.shape[0]
        if payloads is None:
            payloads = np.empty((n, analyser.payload_len()), dtype=np.uint8)
        if pair_done_ns is None:
            pair_done_ns = np.zeros(n, dtype=np.int64)
        rid = ctypes.c_int64()
        _check(lib().svpf_server_submit(self._h, super_builder.handle, analyser.handle, frames.ctypes.data, n,
                                        payloads.ctypes.data, pair_done_ns.ctypes.data, ctypes.byref(rid)))
        self._live[rid.value] = (super_builder, analyser, frames, payloads, pair_done_ns)
        return rid.value

    def wait(self, request: int):
        """-> (payloads, pair_done_ns, (arrival, admit, done) ns on the server clock)."""
        t = (ctypes.c_int64 * 3)()
        rc = lib().svpf_server_wait(self._h, request, t)
        keep = self._live.pop(request)
        _check(rc)
        return keep[3], keep[4], (t[0], t[1], t[2])

    def cancel(self, request: int):
        """Withdraws a request that has not been admitted yet (its wait() then raises with
        code SVPF_ECANCELED); an admitted request runs to completion (ValueError)."""
        _check(lib().svpf_server_cancel(self._h, request))

    def stats(self) -> dict:
        a, c, pb, l = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        pa = ctypes.c_int32()
        lib().svpf_server_stats(self._h, ctypes.byref(a), ctypes.byref(c), ctypes.byref(pb), ctypes.byref(pa),
                                ctypes.byref(l))
        return {"admitted": a.value, "completed": c.value, "peak_device_bytes": pb.value, "peak_active": pa.value,
                "kernel_launches": l.value}


def vector_grid(vdata) -> tuple:
    """(motion_w, motion_h) of the motion-vector planes for a vdata header (metadata.rs:211-244)."""
    v = (ctypes.c_int32 * 16)(*vdata)
    mw, mh = ctypes.c_int32(), ctypes.c_int32()
    _check(lib().svpf_vector_grid(v, ctypes.byref(mw), ctypes.byref(mh)))
    return mw.value, mh.value


def vector_planes_device(vdata, payloads_ptr: int, payload_len: int, npayloads: int, frame_w: int, frame_h: int,
                         planes_ptr: int, status_ptr: int, raw: bool = False, stream: int = 0):
    """decode_vectors + vector_planes on device buffers (see include/svpflow_b200.h)."""
    v = (ctypes.c_int32 * 16)(*vdata)
    _check(lib().svpf_vector_planes_device(v, payloads_ptr, payload_len, npayloads, frame_w, frame_h, int(raw),
                                           planes_ptr, status_ptr, stream))


def scene_class_device(vdata, payloads_ptr: int, payload_len: int, npayloads: int, classes_ptr: int, status_ptr: int,
                       gamma: float = 1.5, blocks: int = 20, zero: int = 200, m1: int = 1600, m2: int = 2800,
                       scene: int = 4000, stream: int = 0):
    """SmoothFps's scene class (int32 per payload, -1 where it does not decode) on device buffers;
    see svpf_scene_class_device."""
    v = (ctypes.c_int32 * 16)(*vdata)
    lim = SceneLimits(int(blocks), int(zero), int(m1), int(m2), int(scene))
    _check(lib().svpf_scene_class_device(v, payloads_ptr, payload_len, npayloads, float(gamma), ctypes.byref(lim),
                                         classes_ptr, status_ptr, stream))


def render_masks_scratch(vdata, npayloads: int) -> int:
    """Bytes of device scratch render_masks_device needs for `npayloads` payloads."""
    v = (ctypes.c_int32 * 16)(*vdata)
    n = lib().svpf_render_masks_scratch(v, int(npayloads))
    if n < 0:
        raise ValueError(lib().svpf_last_error().decode(errors="replace"))
    return n


def render_masks_device(vdata, payloads_ptr: int, payload_len: int, npayloads: int, phase: int, masks_ptr: int,
                        scratch_ptr: int, status_ptr: int, cover: int = 100, area_scale: float = 1.0,
                        area_sharp: float = 1.0, stream: int = 0):
    """SmoothFps's mask planes (cover0 | cover1 | area0 | area1 | area_max per payload, motion-grid
    sized bytes) for the frame at `phase` on device buffers; see svpf_render_masks_device."""
    v = (ctypes.c_int32 * 16)(*vdata)
    _check(lib().svpf_render_masks_device(v, payloads_ptr, payload_len, npayloads, int(phase), int(cover),
                                          float(area_scale), float(area_sharp), masks_ptr, scratch_ptr, status_ptr,
                                          stream))


def render_warp_device(cfg: dict, threshold: int, mode1: bool, interp: bool, src_ptrs, src_strides, src_lens,
                       src_shift: int, motion_x_ptr: int, motion_y_ptr: int, dst_ptrs, dst_strides, stream: int = 0,
                       mask_ptr: int = 0):
    """SmoothFps's single-warp render (algorithms 1 / 2, with or without the mode's mask) of one
    frame's three planes on the device; see svpf_render_warp_device."""
    c = RenderConfig(**{k: int(cfg[k]) for k, _ in RenderConfig._fields_})
    arr = lambda t, v: (t * 3)(*[int(x) for x in v])
    _check(lib().svpf_render_warp_device(ctypes.byref(c), int(threshold), int(mode1), int(interp),
                                         arr(_VP, src_ptrs), arr(ctypes.c_int64, src_strides),
                                         arr(ctypes.c_int64, src_lens), int(src_shift), motion_x_ptr, motion_y_ptr,
                                         mask_ptr or None, arr(_VP, dst_ptrs), arr(ctypes.c_int64, dst_strides),
                                         stream))


def render_blend_device(cfg: dict, threshold: int, mode13: bool, interp: bool, zero_origin: bool, src0_ptrs,
                        src0_strides, src0_lens, src1_ptrs, src1_strides, src1_lens, src_shift: int, motion0,
                        motion1, dst_ptrs, dst_strides, masks=None, stream: int = 0):
    """SmoothFps's two-source blend (algorithms 11 / 13) of one frame's three planes on the device;
    motion0 / motion1 = (x_ptr, y_ptr) device planes, masks = None or (a_ptr, b_ptr); see
    svpf_render_blend_device."""
    c = RenderConfig(**{k: int(cfg[k]) for k, _ in RenderConfig._fields_})
    arr = lambda t, v: (t * 3)(*[int(x) for x in v])
    ma, mb = masks if masks else (None, None)
    _check(lib().svpf_render_blend_device(ctypes.byref(c), int(threshold), int(mode13), int(interp), int(zero_origin),
                                          arr(_VP, src0_ptrs), arr(ctypes.c_int64, src0_strides),
                                          arr(ctypes.c_int64, src0_lens), arr(_VP, src1_ptrs),
                                          arr(ctypes.c_int64, src1_strides), arr(ctypes.c_int64, src1_lens),
                                          int(src_shift), motion0[0], motion0[1], motion1[0], motion1[1], ma, mb,
                                          arr(_VP, dst_ptrs), arr(ctypes.c_int64, dst_strides), stream))


def render_masked_device(cfg: dict, threshold: int, mask_scale: float, mode22: bool, interp: bool, src0_ptrs,
                         src0_strides, src0_lens, src1_ptrs, src1_strides, src1_lens, src_shift: int, motion0,
                         motion1, masks, final_mask_ptr, dst_ptrs, dst_strides, stream: int = 0):
    """SmoothFps's masked two-source blends (algorithms 21 / 22) of one frame on the device; masks =
    (a_ptr, b_ptr), final_mask_ptr 0 or a device plane; see svpf_render_masked_device."""
    c = RenderConfig(**{k: int(cfg[k]) for k, _ in RenderConfig._fields_})
    arr = lambda t, v: (t * 3)(*[int(x) for x in v])
    _check(lib().svpf_render_masked_device(ctypes.byref(c), int(threshold), float(mask_scale), int(mode22),
                                           int(interp), arr(_VP, src0_ptrs), arr(ctypes.c_int64, src0_strides),
                                           arr(ctypes.c_int64, src0_lens), arr(_VP, src1_ptrs),
                                           arr(ctypes.c_int64, src1_strides), arr(ctypes.c_int64, src1_lens),
                                           int(src_shift), motion0[0], motion0[1], motion1[0], motion1[1], masks[0],
                                           masks[1], final_mask_ptr or None, arr(_VP, dst_ptrs),
                                           arr(ctypes.c_int64, dst_strides), stream))


def render_mode23_device(cfg: dict, threshold: int, interp: bool, src0_ptrs, src0_strides, src0_lens, src1_ptrs,
                         src1_strides, src1_lens, src_shift: int, motions, masks, final_mask_ptr, dst_ptrs,
                         dst_strides, stream: int = 0):
    """SmoothFps's algorithm 23 (four motion sets: base0, base1, next0, prev1 as (x_ptr, y_ptr)) of one
    frame on the device; masks = (a_ptr, b_ptr); see svpf_render_mode23_device."""
    c = RenderConfig(**{k: int(cfg[k]) for k, _ in RenderConfig._fields_})
    arr = lambda t, v: (t * 3)(*[int(x) for x in v])
    mx = (_VP * 4)(*[m[0] for m in motions])
    my = (_VP * 4)(*[m[1] for m in motions])
    _check(lib().svpf_render_mode23_device(ctypes.byref(c), int(threshold), int(interp), arr(_VP, src0_ptrs),
                                           arr(ctypes.c_int64, src0_strides), arr(ctypes.c_int64, src0_lens),
                                           arr(_VP, src1_ptrs), arr(ctypes.c_int64, src1_strides),
                                           arr(ctypes.c_int64, src1_lens), int(src_shift), mx, my, masks[0], masks[1],
                                           final_mask_ptr or None, arr(_VP, dst_ptrs), arr(ctypes.c_int64, dst_strides),
                                           stream))
