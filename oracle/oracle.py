"""ctypes front end of the CPU oracle (oracle/svpf_oracle.c) -- TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline / reference leg use
this module: it is the checker, never the product. PARITY UNPINNED: the Rust reference
cannot be built in this image and ships no golden vectors (see svpf_oracle.h).

It also holds `parse_opt`, a restatement of the reference's lenient opt parser
(crates/svpflow-core/src/params.rs:1-450), used to turn an opt string into the looked-up
values the C restatement of SuperOpts/AnalyseOpts::from_opt consumes.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from typing import Any, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libsvpf_oracle.so")


# --------------------------------------------------------------------------- parser
class Obj(list):
    """JSON-ish object: ordered (key, value) members; the LAST duplicate wins (params.rs:77-85)."""

    def get(self, key):  # type: ignore[override]
        for k, v in reversed(self):
            if k == key:
                return v
        return None


class Arr(list):
    pass


class _Null:
    def __repr__(self):
        return "null"


NULL = _Null()


class ParseError(ValueError):
    pass


def parse_opt(text):
    """params::parse (params.rs:1-11): returns the value tree or raises ParseError."""
    b = text.encode() if isinstance(text, str) else bytes(text)
    p = _Parser(b)
    p.skip_ws()
    v = p.value()
    p.skip_ws()
    if p.pos == len(b) or isinstance(v, Obj):
        return v
    raise ParseError("extra data after JSON value")


class _Parser:
    def __init__(self, b):
        self.b = b
        self.pos = 0

    def peek(self):
        return self.b[self.pos] if self.pos < len(self.b) else None

    def at2(self, t):
        return self.b[self.pos:self.pos + 2] == t

    def consume(self, c):
        if self.peek() == c:
            self.pos += 1
            return True
        return False

    def skip_space(self):
        while self.peek() in (0x20, 0x0A, 0x0D, 0x09):
            self.pos += 1

    def skip_ws(self):
        while True:
            self.skip_space()
            if self.at2(b"//"):
                self.pos += 2
                while self.peek() not in (None, 0x0A, 0x0D):
                    self.pos += 1
            elif self.at2(b"/*"):
                self.pos += 2
                while not self.at2(b"*/"):
                    if self.peek() is None:
                        return
                    self.pos += 1
                self.pos += 2
            else:
                return

    def skip_member_space(self):
        self.skip_space()
        if self.at2(b"//") or self.at2(b"/*"):
            raise ParseError("Missing '}' or object member name")

    def value(self):
        self.skip_ws()
        c = self.peek()
        if c == ord("{"):
            return self.obj()
        if c == ord("["):
            return self.arr()
        if c == ord('"'):
            return self.string()
        if c is not None and (c == ord("-") or 48 <= c <= 57):
            return self.number()
        for lit, val in ((b"true", True), (b"false", False), (b"null", NULL)):
            if c == lit[0]:
                if self.b[self.pos:self.pos + len(lit)] == lit:
                    self.pos += len(lit)
                    return val
                raise ParseError("invalid literal")
        raise ParseError("Syntax error: value, object or array expected.")

    def obj(self):
        self.pos += 1
        self.skip_ws()
        out = Obj()
        if self.consume(ord("}")):
            return out
        while True:
            self.skip_member_space()
            if self.peek() == ord('"'):
                key = self.string()
            else:
                key = self.ident()
            self.skip_ws()
            if not self.consume(ord(":")):
                raise ParseError("Missing ':' after object member name")
            out.append((key, self.value()))
            self.skip_ws()
            if self.consume(ord("}")):
                return out
            if not self.consume(ord(",")):
                raise ParseError("Missing ',' or '}' in object declaration")

    def arr(self):
        self.pos += 1
        self.skip_ws()
        out = Arr()
        if self.consume(ord("]")):
            return out
        while True:
            out.append(self.value())
            self.skip_ws()
            if self.consume(ord("]")):
                return out
            if not self.consume(ord(",")):
                raise ParseError("unexpected token")

    def ident(self):
        st = self.pos
        c = self.peek()
        if c is None or not (chr(c).isascii() and (chr(c).isalpha() or c == ord("_"))):
            raise ParseError("Missing '}' or object member name")
        self.pos += 1
        while True:
            c = self.peek()
            if c is not None and chr(c).isascii() and (chr(c).isalnum() or c == ord("_")):
                self.pos += 1
            else:
                break
        return self.b[st:self.pos].decode()

    def string(self):
        self.pos += 1
        out = bytearray()
        while self.pos < len(self.b):
            c = self.b[self.pos]
            self.pos += 1
            if c == ord('"'):
                return out.decode("utf-8", errors="replace")
            if c != ord("\\"):
                out.append(c)
                continue
            e = self.peek()
            if e is not None:
                self.pos += 1
            simple = {ord('"'): b'"', ord("\\"): b"\\", ord("/"): b"/", ord("b"): b"\b", ord("f"): b"\f",
                      ord("n"): b"\n", ord("r"): b"\r", ord("t"): b"\t"}
            if e in simple:
                out += simple[e]
            elif e == ord("u"):
                code = self.hex4()
                if 0xD800 <= code <= 0xDBFF:
                    if not (self.consume(ord("\\")) and self.consume(ord("u"))):
                        raise ParseError("surrogate")
                    low = self.hex4()
                    if not 0xDC00 <= low <= 0xDFFF:
                        raise ParseError("surrogate")
                    out += chr(0x10000 + ((code - 0xD800) << 10) + (low - 0xDC00)).encode()
                elif 0xDC00 <= code <= 0xDFFF:
                    out += "�".encode()
                else:
                    out += chr(code).encode()
            else:
                raise ParseError("Bad escape sequence in string")
        raise ParseError("unterminated string")

    def hex4(self):
        code = 0
        for _ in range(4):
            c = self.peek()
            if c is None or chr(c) not in "0123456789abcdefABCDEF":
                raise ParseError("hex digit expected")
            self.pos += 1
            code = code * 16 + int(chr(c), 16)
        return code

    def digits(self):
        st = self.pos
        while self.peek() is not None and 48 <= self.peek() <= 57:
            self.pos += 1
        return self.pos != st

    def number(self):
        st = self.pos
        neg = self.consume(ord("-"))
        lead = False
        c = self.peek()
        if c is not None and 48 <= c <= 57:
            self.pos += 1
            self.digits()
        elif neg and self.consume(ord(".")):
            if not self.digits():
                raise ParseError("not a number")
            lead = True
        elif neg:
            return 0.0
        else:
            raise ParseError("invalid number")
        if not lead and self.consume(ord(".")):
            self.digits()
        if self.consume(ord("e")) or self.consume(ord("E")):
            if not self.consume(ord("+")):
                self.consume(ord("-"))
            if not self.digits():
                raise ParseError("not a number")
        text = self.b[st:self.pos].decode()
        if lead:
            text = "-0" + text[1:]
        return float(text)


def lookup(tree, path):
    """Value::at (params.rs:69-75)."""
    v = tree
    for k in path:
        if not isinstance(v, Obj):
            return None
        v = v.get(k)
        if v is None:
            return None
    return v


# key paths of the C oracle (svpf_oracle.h OK_*), in enum order
KEYS = [
    ("pel",), ("gpu",), ("scale", "down"), ("scale", "up"), ("full",), ("rc",),
    ("vectors",), ("block", "w"), ("block", "h"), ("block", "overlap"), ("special", "delta"), ("delta",),
    ("main", "penalty", "lambda"), ("penalty", "lambda"),
    ("main", "penalty", "lsad"), ("penalty", "lsad"),
    ("main", "penalty", "plevel"), ("penalty", "plevel"),
    ("main", "penalty", "pnew"), ("penalty", "pnew"),
    ("main", "penalty", "pglobal"), ("penalty", "pglobal"),
    ("main", "penalty", "pzero"), ("penalty", "pzero"),
    ("main", "penalty", "pnbour"), ("penalty", "pnbour"),
    ("main", "penalty", "prev"), ("penalty", "prev"),
    ("main", "search", "type"), ("search", "type"),
    ("main", "search", "distance"), ("search", "distance"),
    ("main", "search", "coarse", "type"), ("search", "coarse", "type"),
    ("main", "search", "coarse", "distance"), ("search", "coarse", "distance"),
    ("main", "search", "coarse", "trymany"), ("search", "coarse", "trymany"),
    ("main", "search", "coarse", "bad", "sad"), ("search", "coarse", "bad", "sad"),
    ("main", "search", "coarse", "bad", "range"),
    ("main", "search", "satd"), ("search", "satd"),
    ("main", "search", "coarse", "satd"),
    ("main", "search", "sort"), ("sort",),
    "REFINE0", ("REFINE0", "thsad"), ("REFINE0", "search", "type"), ("REFINE0", "search", "distance"),
    ("REFINE0", "search", "satd"),
    ("main", "levels"),
]
OR_ABSENT, OR_NUMBER, OR_BOOL, OR_NULL, OR_STRING, OR_ARRAY, OR_OBJECT = range(7)


class OrVal(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("nonempty", ctypes.c_int32), ("num", ctypes.c_double)]


def _val(v) -> tuple:
    if v is None:
        return (OR_ABSENT, 0, 0.0)
    if v is NULL:
        return (OR_NULL, 0, 0.0)
    if isinstance(v, bool):
        return (OR_BOOL, 0, 1.0 if v else 0.0)
    if isinstance(v, float):
        return (OR_NUMBER, 0, v)
    if isinstance(v, str):
        return (OR_STRING, int(len(v) > 0), 0.0)
    if isinstance(v, Arr):
        return (OR_ARRAY, int(len(v) > 0), 0.0)
    if isinstance(v, Obj):
        return (OR_OBJECT, int(len(v) > 0), 0.0)
    raise TypeError(v)


def raw_values(opt: Optional[str]):
    """Array of OrVal for svpf_oracle's from_opt functions (None / parse error -> absent)."""
    arr = (OrVal * len(KEYS))()
    tree = None
    if opt is not None:
        try:
            tree = parse_opt(opt)
        except ParseError:
            tree = None  # super_filter.rs:120 / analyse_filter.rs:85: params::parse(..).ok()
    refine0 = None
    r = lookup(tree, ("refine",)) if tree is not None else None
    if isinstance(r, Arr) and len(r) > 0:
        refine0 = r[0]
    for i, k in enumerate(KEYS):
        if tree is None:
            v = None
        elif k == "REFINE0":
            v = refine0
        elif k[0] == "REFINE0":
            v = lookup(refine0, k[1:]) if refine0 is not None else None
        else:
            v = lookup(tree, k)
        arr[i].kind, arr[i].nonempty, arr[i].num = _val(v)
    return arr


# --------------------------------------------------------------------------- structs
class SuperOpts(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in
                ("pel", "gpu", "scale_down", "scale_up", "full", "rc", "levels", "width", "height")]


class AnalyseOpts(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in
                ("vectors", "block_w", "block_h", "overlap_mode", "overlap_x", "overlap_y", "delta", "pel",
                 "selector", "levels", "super_levels", "width", "height", "lambda_", "lsad")] + \
               [("plevel", ctypes.c_double)] + \
               [(n, ctypes.c_int32) for n in
                ("pnew", "pglobal", "pzero", "pnbour", "prev", "search_type", "coarse_search_type", "distance",
                 "coarse_distance", "coarse_trymany", "coarse_bad_sad", "coarse_bad_range", "fine_satd",
                 "coarse_satd", "has_refine_thsad", "refine_thsad", "refine_search_type", "refine_distance",
                 "refine_satd", "sort")]


class RenderConfig(ctypes.Structure):
    """or_render_config: renderer.rs CpuConfig without the mask scale."""
    _fields_ = [(f, ctypes.c_int32) for f in ("width", "height", "block_w", "block_h", "origin_x", "origin_y",
                                               "grid_w", "grid_h", "chroma_y_div", "source_step")]


class RPlane(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("len", ctypes.c_size_t), ("stride", ctypes.c_size_t),
                ("span", ctypes.c_size_t), ("shift", ctypes.c_uint32)]


class Vec8(ctypes.Structure):
    _fields_ = [("dx", ctypes.c_int16), ("dy", ctypes.c_int16), ("score", ctypes.c_uint32),
                ("luma", ctypes.c_uint8), ("pad", ctypes.c_uint8 * 3)]


class Planes(ctypes.Structure):
    _fields_ = [("y", ctypes.c_void_p), ("y_len", ctypes.c_size_t), ("y_stride", ctypes.c_size_t),
                ("u", ctypes.c_void_p), ("u_len", ctypes.c_size_t), ("u_stride", ctypes.c_size_t),
                ("v", ctypes.c_void_p), ("v_len", ctypes.c_size_t), ("v_stride", ctypes.c_size_t),
                ("luma_w", ctypes.c_size_t), ("luma_h", ctypes.c_size_t),
                ("pel", ctypes.c_int32), ("levels", ctypes.c_int32), ("full", ctypes.c_int32)]


_lib = None


def build():
    """Compiles the oracle with its own Makefile (gcc)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


LIB16_PATH = os.path.join(HERE, "_build", "libsvpf_oracle16.so")
_lib16 = None


def lib16():
    """The same restatement built for uint16 samples (this project's 10-bit extension: values
    0..1023, chroma default 512, block luma byte = mean >> 2; no reference behaviour)."""
    global _lib16
    if _lib16 is None:
        if not os.path.exists(LIB16_PATH):
            build()
        _lib16 = _setup(ctypes.CDLL(LIB16_PATH))
    return _lib16


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = _setup(ctypes.CDLL(LIB_PATH))
    return _lib


def _setup(L):
    """Argument and result types of the restatement's exports."""
    P = ctypes.POINTER
    L.or_super_opts_from_opt.argtypes = [P(OrVal), ctypes.c_int32, ctypes.c_int32, P(SuperOpts), ctypes.c_char_p, ctypes.c_size_t]
    L.or_super_pack_data.restype = ctypes.c_int64
    L.or_super_pack_data.argtypes = [P(SuperOpts)]
    L.or_super_height.argtypes = [P(SuperOpts)]
    L.or_super_output_len.restype = ctypes.c_size_t
    L.or_super_output_len.argtypes = [P(SuperOpts)]
    L.or_analyse_opts_from_opt.argtypes = [P(OrVal), ctypes.c_int64, P(SuperOpts), P(AnalyseOpts), ctypes.c_char_p, ctypes.c_size_t]
    L.or_analyser_portable.argtypes = [P(SuperOpts), ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                       P(AnalyseOpts), ctypes.c_char_p, ctypes.c_size_t]
    L.or_build_super_portable.argtypes = [P(SuperOpts), ctypes.c_void_p, ctypes.c_void_p]
    L.or_build_super_many.argtypes = [P(SuperOpts), P(ctypes.c_void_p), P(ctypes.c_void_p), ctypes.c_int32, ctypes.c_int32]
    L.or_build_plane.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t,
                                 ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t,
                                 ctypes.c_int32, P(SuperOpts)]
    L.or_payload_len.restype = ctypes.c_size_t
    L.or_payload_len.argtypes = [P(AnalyseOpts)]
    L.or_analyse_portable.argtypes = [P(AnalyseOpts), P(SuperOpts), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.or_analyse_clip.argtypes = [P(AnalyseOpts), P(SuperOpts), P(ctypes.c_void_p), ctypes.c_int32, ctypes.c_int32,
                                  ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32]
    L.or_analyse_pair.argtypes = [P(Planes), P(Planes), P(AnalyseOpts), ctypes.c_void_p, ctypes.c_void_p]
    L.or_pack_vdata_header.argtypes = [P(AnalyseOpts), P(ctypes.c_int32)]
    L.or_hadamard4_satd.restype = ctypes.c_uint32
    L.or_vector_grid.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.or_vector_planes.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int32,
                                   ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p]
    L.or_render_masks.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int32, ctypes.c_int32,
                                  ctypes.c_double, ctypes.c_double, ctypes.c_void_p]
    L.or_scene_class.restype = ctypes.c_int32
    L.or_scene_class.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_double] + \
        [ctypes.c_int32] * 5
    L.or_hadamard4_satd.argtypes = [P(ctypes.c_int32)]
    L.or_adapt_lambda.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_uint32]
    L.or_exact_lambda.argtypes = [P(AnalyseOpts), ctypes.c_int32, ctypes.c_int32]
    L.or_rescale_scores.argtypes = [P(Vec8), ctypes.c_size_t, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]
    L.or_global_doubled.argtypes = [P(Vec8), ctypes.c_size_t, P(ctypes.c_int32), P(ctypes.c_int32)]
    L.or_block_cost_lc.argtypes = [P(Planes), P(Planes)] + [ctypes.c_int32] * 9 + [P(ctypes.c_uint32), P(ctypes.c_uint32)]
    L.or_last_counters.argtypes = [P(ctypes.c_uint64)]
    L.or_total_counters.argtypes = [P(ctypes.c_uint64), ctypes.c_int32]
    if hasattr(L, "or_render_luts"):  # the 8-bit build only
        L.or_render_luts.argtypes = [ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p]
        L.or_render_dual_plane.argtypes = [P(RenderConfig)] + [ctypes.c_int32] * 6 + [P(RPlane), P(RPlane)] + \
            [ctypes.c_void_p] * 4 + [ctypes.c_size_t] + [ctypes.c_void_p] * 4 + [ctypes.c_size_t, ctypes.c_size_t]
        L.or_render_mode23_plane.argtypes = [P(RenderConfig)] + [ctypes.c_int32] * 3 + [P(RPlane), P(RPlane)] + \
            [ctypes.c_void_p] * 2 + [ctypes.c_size_t] + [ctypes.c_void_p] * 4 + [ctypes.c_size_t, ctypes.c_size_t]
        L.or_render_threshold_limit.restype = ctypes.c_int32
        L.or_render_threshold_limit.argtypes = [ctypes.c_int32, ctypes.c_double]
        L.or_render_warp_plane.argtypes = [P(RenderConfig), ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p,
                                           P(RPlane), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                           ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t]
    for f in ("or_reduce_dim", "or_auto_levels", "or_super_plane_height", "or_auto_search_levels"):
        getattr(L, f).argtypes = [ctypes.c_int32] * {"or_reduce_dim": 2, "or_auto_levels": 2,
                                                       "or_super_plane_height": 4, "or_auto_search_levels": 6}[f]
    L.or_level_grid.argtypes = [P(AnalyseOpts), ctypes.c_int32, P(ctypes.c_int32), P(ctypes.c_int32)]
    return L


def _err():
    return ctypes.create_string_buffer(512)


def super_opts(width: int, height: int, opt: Optional[str] = None) -> SuperOpts:
    o = SuperOpts()
    e = _err()
    if lib().or_super_opts_from_opt(raw_values(opt), width, height, ctypes.byref(o), e, 512):
        raise ValueError(e.value.decode())
    return o


def super_opts_portable(width: int, height: int, pel: int) -> SuperOpts:
    """SuperBuilder::new (portable.rs:30-62)."""
    if pel not in (1, 2, 4):
        raise ValueError("pel must be 1, 2 or 4")
    if width <= 0 or height <= 0 or width % 2 or height % 2:
        raise ValueError("dimensions must be positive and even")
    o = super_opts(width, height, None)
    o.pel = pel
    return o


def analyse_opts(sdata: int, opt: Optional[str] = None, hint: Optional[SuperOpts] = None,
                 src_width: int = 0, src_height: int = 0) -> AnalyseOpts:
    """AnalyseOpts::from_opt + the src-clip size override of analyse_filter.rs:96-101."""
    o = AnalyseOpts()
    e = _err()
    if lib().or_analyse_opts_from_opt(raw_values(opt), sdata, ctypes.byref(hint) if hint else None,
                                      ctypes.byref(o), e, 512):
        raise ValueError(e.value.decode())
    if src_width > 0:
        o.width = src_width
    if src_height > 0:
        o.height = src_height
    return o


def analyser_portable(so: SuperOpts, bw: int, bh: int, overlap_mode: int, vectors: int) -> AnalyseOpts:
    o = AnalyseOpts()
    e = _err()
    if lib().or_analyser_portable(ctypes.byref(so), bw, bh, overlap_mode, vectors, ctypes.byref(o), e, 512):
        raise ValueError(e.value.decode())
    return o


def sdata(so: SuperOpts) -> int:
    return lib().or_super_pack_data(ctypes.byref(so))


def super_height(so: SuperOpts) -> int:
    return lib().or_super_height(ctypes.byref(so))


def super_output_len(so: SuperOpts) -> int:
    return lib().or_super_output_len(ctypes.byref(so))


def _ptr(a: np.ndarray) -> int:
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def build_super(so: SuperOpts, src: np.ndarray) -> np.ndarray:
    """SuperBuilder::build on one packed I420 frame -> the super frame bytes."""
    src = np.ascontiguousarray(src, dtype=np.uint8)
    out = np.zeros(super_output_len(so), dtype=np.uint8)
    lib().or_build_super_portable(ctypes.byref(so), _ptr(src), _ptr(out))
    return out


def build_super_many(so: SuperOpts, frames: np.ndarray, threads: int = 1) -> np.ndarray:
    frames = np.ascontiguousarray(frames, dtype=np.uint8)
    n = frames.shape[0]
    out = np.zeros((n, super_output_len(so)), dtype=np.uint8)
    srcp = (ctypes.c_void_p * n)(*[frames[i].ctypes.data for i in range(n)])
    dstp = (ctypes.c_void_p * n)(*[out[i].ctypes.data for i in range(n)])
    lib().or_build_super_many(ctypes.byref(so), srcp, dstp, n, threads)
    return out


def payload_len(ao: AnalyseOpts) -> int:
    return lib().or_payload_len(ctypes.byref(ao))


def vdata_header(ao: AnalyseOpts) -> list:
    h = (ctypes.c_int32 * 16)()
    lib().or_pack_vdata_header(ctypes.byref(ao), h)
    return list(h)


def analyse(ao: AnalyseOpts, so: SuperOpts, cur: np.ndarray, ref: np.ndarray) -> np.ndarray:
    """Analyser::analyse on two portable super frames -> payload bytes."""
    out = np.zeros(payload_len(ao), dtype=np.uint8)
    cur = np.ascontiguousarray(cur, dtype=np.uint8)
    ref = np.ascontiguousarray(ref, dtype=np.uint8)
    rc = lib().or_analyse_portable(ctypes.byref(ao), ctypes.byref(so), _ptr(cur), _ptr(ref), _ptr(out))
    if rc:
        raise RuntimeError("the reference panics on this input (index out of range)")
    return out


def counters() -> list:
    """[evaluations, luma samples, chroma samples, luma under SATD, chroma under SATD] of the
    last pair analysed on this thread."""
    c = (ctypes.c_uint64 * 5)()
    lib().or_last_counters(c)
    return list(c)


def total_counters(reset: bool = False, px16: bool = False) -> list:
    """counters() summed over every pair analysed (any thread) since the last reset; px16 reads
    the uint16 build's."""
    c = (ctypes.c_uint64 * 5)()
    (lib16() if px16 else lib()).or_total_counters(c, int(reset))
    return list(c)


def integer_ops(c) -> float:
    """Algorithmic integer operations of the compares counted in `c`: about 2 per sample for SAD
    (absolute difference, accumulate) and 111 per 4x4 tile, 6.94 per sample, for SATD (16
    differences, 64 butterfly adds, 16 absolute values, 15 adds)."""
    satd = c[3] + c[4]
    sad = c[1] + c[2] - satd
    return 2.0 * sad + 111.0 / 16.0 * satd


def analyse_clip(ao: AnalyseOpts, so: SuperOpts, supers: np.ndarray, first: int, count: int,
                 threads: int = 1) -> np.ndarray:
    """Output frames [first, first+count) of a clip of portable super frames."""
    supers = np.ascontiguousarray(supers, dtype=np.uint8)
    n = supers.shape[0]
    pl = payload_len(ao)
    out = np.zeros((count, pl), dtype=np.uint8)
    ptrs = (ctypes.c_void_p * n)(*[supers[i].ctypes.data for i in range(n)])
    rc = lib().or_analyse_clip(ctypes.byref(ao), ctypes.byref(so), ptrs, n, first, count, _ptr(out), threads)
    if rc:
        raise RuntimeError("the reference panics on this input (index out of range)")
    return out


def hadamard4(diff16) -> int:
    a = (ctypes.c_int32 * 16)(*[int(v) for v in diff16])
    return lib().or_hadamard4_satd(a)


def adapt_lambda(nlambda: int, lsad: int, score: int) -> int:
    return lib().or_adapt_lambda(nlambda, lsad, score & 0xFFFFFFFF)


def reduce_dim(d: int, n: int) -> int:
    return lib().or_reduce_dim(d, n)


def auto_levels(w: int, h: int) -> int:
    return lib().or_auto_levels(w, h)


def auto_search_levels(w, h, bw, bh, ox, oy) -> int:
    return lib().or_auto_search_levels(w, h, bw, bh, ox, oy)


def level_grid(ao: AnalyseOpts, level: int):
    gw, gh = ctypes.c_int32(), ctypes.c_int32()
    lib().or_level_grid(ctypes.byref(ao), level, ctypes.byref(gw), ctypes.byref(gh))
    return gw.value, gh.value


def build_super_strided(so: SuperOpts, src: np.ndarray, y_stride: int, c_stride: int) -> np.ndarray:
    """A frame server's Super frame (super_filter.rs:210-262): zeroed planes at the given row
    pitches (Y y_stride x H, then U and V c_stride x H/2), each built by build_plane from
    the packed I420 source. Returned as one buffer Y | U | V."""
    src = np.ascontiguousarray(src, dtype=np.uint8)
    w, h = so.width, so.height
    cw, ch = w // 2, h // 2
    H = super_height(so)
    out = np.zeros(y_stride * H + 2 * c_stride * (H // 2), dtype=np.uint8)
    planes = [(0, y_stride, H, src[: w * h], w, w, h, 0),
              (y_stride * H, c_stride, H // 2, src[w * h: w * h + cw * ch], cw, cw, ch, 1),
              (y_stride * H + c_stride * (H // 2), c_stride, H // 2, src[w * h + cw * ch:], cw, cw, ch, 1)]
    for off, st, rows, s, sst, pw, ph, chroma in planes:
        s = np.ascontiguousarray(s)
        dst = out[off: off + st * rows]
        lib().or_build_plane(_ptr(dst), dst.size, st, _ptr(s), s.size, sst, pw, ph, w, h, chroma, ctypes.byref(so))
    return out


def analyse_strided(ao: AnalyseOpts, cur: np.ndarray, ref: np.ndarray, y_stride: int, c_stride: int) -> np.ndarray:
    """get_frame_analyse's payload (analyse_filter.rs:287-325) for two super frames laid out
    as build_super_strided returns them."""
    y_h = lib().or_super_plane_height(ao.height, ao.pel, ao.super_levels, 1)
    uv_h = y_h // 2
    keep = []

    def planes(buf):
        buf = np.ascontiguousarray(buf, dtype=np.uint8)
        keep.append(buf)
        base = buf.ctypes.data
        yl, cl = y_stride * y_h, c_stride * uv_h
        return Planes(base, yl, y_stride, base + yl, cl, c_stride, base + yl + cl, cl, c_stride,
                      ao.width, ao.height, ao.pel, ao.super_levels, 1)

    pc, pr = planes(cur), planes(ref)
    bw, bh, ox, oy = (ctypes.c_int32() for _ in range(4))
    lib().or_output_block(ctypes.byref(ao), ctypes.byref(bw), ctypes.byref(bh), ctypes.byref(ox), ctypes.byref(oy))
    gw, gh = ctypes.c_int32(), ctypes.c_int32()
    lib().or_grid(ctypes.byref(ao), bw, bh, ox, oy, ctypes.byref(gw), ctypes.byref(gh))
    n = gw.value * gh.value
    bwd, fwd = (Vec8 * n)(), (Vec8 * n)()
    rc = lib().or_analyse_pair(ctypes.byref(pc), ctypes.byref(pr), ctypes.byref(ao),
                               bwd if ao.vectors & 1 else None, fwd if ao.vectors & 2 else None)
    if rc:
        raise RuntimeError("the reference panics on this input (index out of range)")
    out = np.zeros(payload_len(ao), dtype=np.uint8)
    lib().or_pack_vector_frame(ctypes.byref(ao), bwd if ao.vectors & 1 else None, fwd if ao.vectors & 2 else None,
                               _ptr(out))
    return out


def vector_grid(vdata) -> tuple:
    v = (ctypes.c_int32 * 16)(*vdata)
    mw, mh = ctypes.c_int32(), ctypes.c_int32()
    lib().or_vector_grid(v, ctypes.byref(mw), ctypes.byref(mh))
    return mw.value, mh.value


def vector_planes(vdata, payload: np.ndarray, frame_w: int, frame_h: int, raw: bool = False):
    """decode_vectors + vector_planes (svpflow-core) for both sets -> uint16 [4, mh, mw], or None
    when the payload does not decode."""
    mw, mh = vector_grid(vdata)
    out = np.zeros(4 * max(mw, 0) * max(mh, 0), dtype=np.uint16)
    payload = np.ascontiguousarray(payload, dtype=np.uint8)
    v = (ctypes.c_int32 * 16)(*vdata)
    rc = lib().or_vector_planes(v, _ptr(payload), payload.size, frame_w, frame_h, int(raw), out.ctypes.data)
    return None if rc else out.reshape(4, mh, mw)


def render_masks(vdata, payload: np.ndarray, phase: int, cover: int = 100, area_scale: float = 1.0,
                 area_sharp: float = 1.0):
    """SmoothFps' mask planes for one payload at `phase` -> uint8 [5, mh, mw] = cover0, cover1, area0,
    area1, max(area0, area1); None when the payload does not decode."""
    mw, mh = vector_grid(vdata)
    out = np.zeros(5 * max(mw, 0) * max(mh, 0), dtype=np.uint8)
    payload = np.ascontiguousarray(payload, dtype=np.uint8)
    v = (ctypes.c_int32 * 16)(*vdata)
    rc = lib().or_render_masks(v, _ptr(payload), payload.size, int(phase), int(cover), float(area_scale),
                               float(area_sharp), out.ctypes.data)
    return None if rc else out.reshape(5, mh, mw)


def scene_class(vdata, payload: np.ndarray, gamma: float = 1.5, blocks: int = 20, zero: int = 200, m1: int = 1600,
                m2: int = 2800, scene: int = 4000) -> int:
    """SmoothFps's scene class (0..3) of one payload; -1 when it does not decode. Defaults: the
    scene.luma gamma and the scene limits SmoothFps uses in its default mode."""
    payload = np.ascontiguousarray(payload, dtype=np.uint8)
    v = (ctypes.c_int32 * 16)(*vdata)
    return lib().or_scene_class(v, _ptr(payload), payload.size, float(gamma), int(blocks), int(zero), int(m1),
                                int(m2), int(scene))


# ---- 10-bit extension (uint16 samples), same options as the 8-bit path
def build_super16(so: SuperOpts, src: np.ndarray) -> np.ndarray:
    src = np.ascontiguousarray(src, dtype=np.uint16)
    out = np.zeros(super_output_len(so), dtype=np.uint16)
    lib16().or_build_super_portable(ctypes.byref(so), _ptr(src), _ptr(out))
    return out


def build_super_many16(so: SuperOpts, frames: np.ndarray, threads: int = 1) -> np.ndarray:
    frames = np.ascontiguousarray(frames, dtype=np.uint16)
    n = frames.shape[0]
    out = np.zeros((n, super_output_len(so)), dtype=np.uint16)
    srcp = (ctypes.c_void_p * n)(*[frames[i].ctypes.data for i in range(n)])
    dstp = (ctypes.c_void_p * n)(*[out[i].ctypes.data for i in range(n)])
    lib16().or_build_super_many(ctypes.byref(so), srcp, dstp, n, threads)
    return out


def analyse_clip16(ao: AnalyseOpts, so: SuperOpts, supers: np.ndarray, first: int, count: int,
                   threads: int = 1) -> np.ndarray:
    supers = np.ascontiguousarray(supers, dtype=np.uint16)
    n = supers.shape[0]
    out = np.zeros((count, payload_len(ao)), dtype=np.uint8)
    ptrs = (ctypes.c_void_p * n)(*[supers[i].ctypes.data for i in range(n)])
    rc = lib16().or_analyse_clip(ctypes.byref(ao), ctypes.byref(so), ptrs, n, first, count, _ptr(out), threads)
    if rc:
        raise RuntimeError("the search indexes out of range on this input (the reference's panic)")
    return out


# ---- SmoothFps single-warp render (renderer.rs render_mode1_or_2 without masks)
def render_luts(threshold: int):
    """CpuRenderer::set_threshold: (inverse_lut, threshold_lut), int16[2048] each."""
    inv = np.zeros(2048, dtype=np.int16)
    thr = np.zeros(2048, dtype=np.int16)
    lib().or_render_luts(int(threshold), _ptr(inv), _ptr(thr))
    return inv, thr


def render_warp_plane(cfg: dict, chroma: bool, interp: bool, lut: np.ndarray, src: np.ndarray, src_stride: int,
                      src_span: int, src_shift: int, mx: np.ndarray, my: np.ndarray, dst_stride: int,
                      dst_rows: int, mask: np.ndarray = None) -> np.ndarray:
    """render_selected_warp_rows over a whole plane: uint8 [dst_rows, dst_stride] (bytes the reference
    leaves untouched stay 0)."""
    c = RenderConfig(**{k: int(cfg[k]) for k, _ in RenderConfig._fields_})
    src = np.ascontiguousarray(src, dtype=np.uint8).reshape(-1)
    mx = np.ascontiguousarray(mx, dtype=np.uint16).reshape(-1)
    my = np.ascontiguousarray(my, dtype=np.uint16).reshape(-1)
    lut = np.ascontiguousarray(lut, dtype=np.int16)
    assert mx.size == my.size and lut.size == 2048
    pl = RPlane(src.ctypes.data, src.size, src_stride, src_span, src_shift)
    dst = np.zeros(dst_rows * dst_stride, dtype=np.uint8)
    mk = None
    if mask is not None:
        mk = np.ascontiguousarray(mask, dtype=np.uint8).reshape(-1)
        assert mk.size == mx.size
    lib().or_render_warp_plane(ctypes.byref(c), int(chroma), int(interp), _ptr(lut), ctypes.byref(pl), _ptr(mx),
                               _ptr(my), mx.size, None if mk is None else _ptr(mk), _ptr(dst), dst_stride, dst.size)
    return dst.reshape(dst_rows, dst_stride)


def render_threshold_limit(threshold: int, scale: float) -> int:
    return lib().or_render_threshold_limit(int(threshold), float(scale))


def render_dual_plane(cfg: dict, chroma: bool, interp: bool, zero_origin: bool, mode: int, threshold: int,
                      srcs, strides, spans, shift: int, motion0, motion1, dst_stride: int, dst_rows: int,
                      masks=None, final_mask=None, threshold_limit: int = 0) -> np.ndarray:
    """render_mode11_or_13 / render_mode21_or_22 for one plane: srcs / strides / spans of sources 0
    and 1, motion0 / motion1 = (mx, my) of the two sets, masks = (a, b) or None, final_mask for 21 / 22."""
    c = RenderConfig(**{k: int(cfg[k]) for k, _ in RenderConfig._fields_})
    ss = [np.ascontiguousarray(x, dtype=np.uint8).reshape(-1) for x in srcs]
    pls = [RPlane(ss[i].ctypes.data, ss[i].size, strides[i], spans[i], shift) for i in range(2)]
    ms = [np.ascontiguousarray(m, dtype=np.uint16).reshape(-1) for m in (*motion0, *motion1)]
    n = ms[0].size
    mk = [None if m is None else np.ascontiguousarray(m, dtype=np.uint8).reshape(-1)
          for m in ((masks or (None, None))[0], (masks or (None, None))[1], final_mask)]
    dst = np.zeros(dst_rows * dst_stride, dtype=np.uint8)
    lib().or_render_dual_plane(ctypes.byref(c), int(chroma), int(interp), int(zero_origin), int(mode),
                               int(threshold), int(threshold_limit), ctypes.byref(pls[0]), ctypes.byref(pls[1]),
                               *[_ptr(m) for m in ms], n, *[None if m is None else _ptr(m) for m in mk], _ptr(dst),
                               dst_stride, dst.size)
    return dst.reshape(dst_rows, dst_stride)


def render_mode23_plane(cfg: dict, chroma: bool, interp: bool, threshold: int, srcs, strides, spans, shift: int,
                        motions, masks, final_mask, dst_stride: int, dst_rows: int) -> np.ndarray:
    """render_mode23 for one plane: motions = 4 (mx, my) sets (base0, base1, next0, prev1), masks = (a, b)."""
    c = RenderConfig(**{k: int(cfg[k]) for k, _ in RenderConfig._fields_})
    ss = [np.ascontiguousarray(x, dtype=np.uint8).reshape(-1) for x in srcs]
    pls = [RPlane(ss[i].ctypes.data, ss[i].size, strides[i], spans[i], shift) for i in range(2)]
    mx = [np.ascontiguousarray(m[0], dtype=np.uint16).reshape(-1) for m in motions]
    my = [np.ascontiguousarray(m[1], dtype=np.uint16).reshape(-1) for m in motions]
    px_ = (ctypes.c_void_p * 4)(*[m.ctypes.data for m in mx])
    py_ = (ctypes.c_void_p * 4)(*[m.ctypes.data for m in my])
    mk = [None if m is None else np.ascontiguousarray(m, dtype=np.uint8).reshape(-1) for m in (*masks, final_mask)]
    dst = np.zeros(dst_rows * dst_stride, dtype=np.uint8)
    lib().or_render_mode23_plane(ctypes.byref(c), int(chroma), int(interp), int(threshold), ctypes.byref(pls[0]),
                                 ctypes.byref(pls[1]), px_, py_, mx[0].size,
                                 *[None if m is None else _ptr(m) for m in mk], _ptr(dst), dst_stride, dst.size)
    return dst.reshape(dst_rows, dst_stride)
