"""Second, independent restatement of the reference path in pure Python (small inputs only).

TEST INFRASTRUCTURE: it exists to cross-check oracle/svpf_oracle.c (differential testing of
two restatements), because the Rust reference cannot run here and has no golden vectors
(parity unpinned). Written from crates/svpflow1/src/{super_opts,super_build,analyse_opts,
analyse_search,portable}.rs directly, with Python integers and explicit wrapping where the
reference's release build wraps (usize, i32) or saturates.
"""
from __future__ import annotations

import math
import struct

from .oracle import Arr, NULL, Obj, ParseError, lookup, parse_opt

U64 = (1 << 64) - 1
U32 = (1 << 32) - 1
I32MAX, I32MIN = (1 << 31) - 1, -(1 << 31)
I64MAX = (1 << 63) - 1
# sample width: 8-bit as the reference; set_sample_bits(10) gives this project's 10-bit extension
# (uint16 samples: clamps at 1023, chroma default 512, payload block luma = mean >> 2)
PX_MAX, PX_MID, DC_SHIFT = 255, 128, 0


def set_sample_bits(bits: int):
    global PX_MAX, PX_MID, DC_SHIFT
    PX_MAX, PX_MID, DC_SHIFT = (1023, 512, 2) if bits > 8 else (255, 128, 0)


def us(v):  # `i32 as usize` / wrapping usize arithmetic
    return v & U64


def get(buf, i, d):  # slice.get(i).copied().unwrap_or(d)
    return buf[i] if 0 <= i < len(buf) else d


def sat_u32(v):
    return U32 if v > U32 else v


def sat_i32(v):
    return I32MAX if v > I32MAX else (I32MIN if v < I32MIN else v)


def as_i32(v):  # i64 as i32 (wrapping)
    v &= U32
    return v - (1 << 32) if v >= (1 << 31) else v


def f64_as_i32(x):
    if x != x:
        return 0
    if x >= 2147483647.0:
        return I32MAX
    if x <= -2147483648.0:
        return I32MIN
    return int(x)


def i16(v):
    v &= 0xFFFF
    return v - 0x10000 if v >= 0x8000 else v


def avg(a, b):
    return (a + b + 1) >> 1


def clamp(v, lo, hi):
    return lo if v < lo else (hi if v > hi else v)


def tdiv(a, b):  # Rust integer division (truncation toward zero)
    q = abs(a) // abs(b)
    return q if (a >= 0) == (b >= 0) else -q


# ------------------------------------------------------------------ params lookups (params.rs:23-53)
def int_at(tree, path):
    v = lookup(tree, path) if tree is not None else None
    if isinstance(v, bool):
        return int(v)
    if isinstance(v, float):
        if not math.isfinite(v):
            return None
        t = math.trunc(v)
        return t if -(1 << 63) <= t < (1 << 63) else None
    if v is NULL:
        return 0
    return None


def bool_at(tree, path):
    v = lookup(tree, path) if tree is not None else None
    if v is None:
        return None
    if isinstance(v, bool):
        return v
    if isinstance(v, float):
        return v != 0.0
    if isinstance(v, (str, Arr, Obj)):
        return len(v) > 0
    if v is NULL:
        return False
    return None


def float_at(tree, path):
    v = lookup(tree, path) if tree is not None else None
    if isinstance(v, bool):
        return float(int(v))
    if isinstance(v, float):
        return v
    if v is NULL:
        return 0.0
    return None


def first(*vals):
    for v in vals:
        if v is not None:
            return v
    return None


def tree_of(opt):
    if opt is None:
        return None
    try:
        return parse_opt(opt)
    except ParseError:
        return None


# ------------------------------------------------------------------ super_opts.rs
def reduce_dim(dim, n):
    for _ in range(n):
        dim = 2 * tdiv(dim, 4)
    return dim


def auto_levels(w, h):
    i = 0
    while True:
        if reduce_dim(h, i) < 4 or reduce_dim(w, i) < 4:
            return i
        i += 1


def super_plane_height(base_h, pel, levels, full):
    total = pel * pel * base_h if full else 0
    for lv in range(1, levels):
        total += reduce_dim(base_h, lv)
    return total


class SuperOpts:
    pass


def super_from_opt(opt, w, h):
    t = tree_of(opt)
    o = SuperOpts()
    pel = as_i32(first(int_at(t, ("pel",)), 2))
    if pel not in (1, 2, 4):
        raise ValueError("SVSuper: pel has to be 1 or 2 or 4")
    gpu = as_i32(first(int_at(t, ("gpu",)), 1))
    if not 0 <= gpu <= 2:
        raise ValueError("SVSuper: gpu has to be 0 or 1 or 2")
    o.scale_down = as_i32(first(int_at(t, ("scale", "down")), 4))
    o.scale_up = as_i32(first(int_at(t, ("scale", "up")), 2))
    if gpu != 0:
        o.scale_up = 0
    o.full = first(bool_at(t, ("full",)), True)
    if pel >= 2 and not o.full:
        raise ValueError("SVSuper: can't ignore finest level with high pel value")
    o.rc = first(bool_at(t, ("rc",)), False)
    o.pel, o.gpu, o.levels, o.width, o.height = pel, gpu, auto_levels(w, h), w, h
    return o


def pack_data(o):
    flags = (1 if o.rc else 0) | (0 if o.full else 2)
    raw = (o.height & 0xFFFF) | ((o.width & 0xFFFF) << 16) | ((o.pel & 0xFF) << 32) | ((o.levels & 0xFF) << 40) \
        | ((o.gpu & 0xFF) << 48) | (flags << 56)
    return raw - (1 << 64) if raw >= (1 << 63) else raw


# ------------------------------------------------------------------ super_build.rs
def build_plane(dst, dst_stride, src, src_stride, src_w, src_h, luma_w, luma_h, chroma, o):
    levels, pel = o.levels, o.pel
    if levels == 0 or src_w == 0 or src_h == 0:
        return

    def size(lv):
        yw, yh = reduce_dim(luma_w, lv), reduce_dim(luma_h, lv)
        return (yw // 2, yh // 2) if chroma else (yw, yh)

    level_y, y = [], 0
    for lv in range(levels):
        level_y.append(y)
        y += size(lv)[1] * (pel * pel if lv == 0 and o.full else 1)
    bw, bh = size(0)
    n_dst = len(dst)
    for row in range(min(bh, src_h)):
        do, so = (level_y[0] + row) * dst_stride, row * src_stride
        n = min(bw, src_w, max(n_dst - do, 0), max(len(src) - so, 0))
        if n > 0:
            dst[do:do + n] = src[so:so + n]
        if bw > 0 and dst_stride > bw:
            e = dst[do + bw - 1]
            for p in range(bw, dst_stride):
                if do + p < n_dst:
                    dst[do + p] = e
    if o.scale_down == 4:
        for lv in range(levels - 1):
            sw, sh = size(lv)
            dw, dh = size(lv + 1)
            _reduce(dst, dst_stride, level_y[lv + 1], dw, dh, level_y[lv], sw, sh)
    if pel >= 2 and o.gpu <= 1 and o.full:
        if o.scale_up == 0:
            _bilinear(dst, dst_stride, level_y[0], bw, bh)
        elif o.scale_up == 2:
            _bicubic(dst, dst_stride, level_y[0], bw, bh)


def _reduce(buf, stride, drow0, dw, dh, srow0, sw, sh):
    if dw == 0 or dh == 0 or sw == 0 or sh == 0:
        return
    smp = lambda y, x: get(buf, (srow0 + y) * stride + x, 0)
    rows = []
    for dy in range(dh):
        sy = 2 * dy
        if dy == 0 or dy + 1 == dh or sy - 2 < 0 or sy + 3 >= sh:
            y0, y1 = min(sy, max(sh - 1, 0)), min(sy + 1, max(sh - 1, 0))
            rows.append([avg(smp(y0, x), smp(y1, x)) for x in range(sw)])
        else:
            st = sy - 2
            rows.append([min((smp(st, x) + smp(st + 5, x) + 5 * (smp(st + 1, x) + smp(st + 4, x))
                              + 10 * (smp(st + 2, x) + smp(st + 3, x)) + 16) >> 5, PX_MAX) for x in range(sw)])
    for dy in range(dh):
        row = rows[dy]
        _h6(row, dw)
        base = (drow0 + dy) * stride
        n = min(sw, max(len(buf) - base, 0))
        buf[base:base + n] = row[:n]


def _h6(row, dw):
    g = lambda a, i, d: a[i] if 0 <= i < len(a) else d
    if dw == 0 or not row:
        return
    if dw <= 2:
        for i in range(dw):
            a = g(row, 2 * i, 0)
            row[i] = avg(a, g(row, 2 * i + 1, a))
        return
    src = list(row)
    n = len(src)
    row[0] = avg(src[0], g(src, 1, src[0]))
    left = row[0]
    for i in range(max(dw - 2, 0)):
        k = 5 + 2 * i
        pk = src[k] if k < n else src[n - 1]
        v = (left + pk + 10 * (g(src, k - 3, 0) + g(src, k - 2, 0)) + 5 * (g(src, k - 4, 0) + g(src, (k - 1) & ~1, 0))
             + 16) >> 5
        row[i + 1] = min(v, PX_MAX)
        left = g(src, k - 3, 0)
    for i in range(max(dw - 1, 1), dw):
        a = g(src, 2 * i, 0)
        row[i] = avg(a, g(src, 2 * i + 1, a))


def _bilinear(d, s, r0, w, h):
    H, V, HV = r0 + h, r0 + 2 * h, r0 + 3 * h
    L = len(d)
    for y in range(h):
        for x in range(w):
            a = get(d, (r0 + y) * s + x, 0)
            b = get(d, (r0 + y) * s + x + 1, a)
            if (H + y) * s + x < L:
                d[(H + y) * s + x] = avg(a, b)
    for y in range(h):
        for x in range(w):
            a = get(d, (r0 + y) * s + x, 0)
            b = get(d, (r0 + y + 1) * s + x, a)
            if (V + y) * s + x < L:
                d[(V + y) * s + x] = avg(a, b)
    n = min(w, max(L - V * s, 0), max(L - r0 * s, 0))
    d[V * s:V * s + n] = d[r0 * s:r0 * s + n]
    for y in range(h):
        for x in range(w):
            a = get(d, (r0 + y) * s + x, 0)
            b = get(d, (r0 + y + 1) * s + 1 + x, a)
            if (HV + y) * s + x < L:
                d[(HV + y) * s + x] = avg(a, b)
    n = min(w, max(L - HV * s, 0), max(L - (r0 * s + 1), 0))
    d[HV * s:HV * s + n] = d[r0 * s + 1:r0 * s + 1 + n]


def _half(b, i, step, p, n):
    if p < 2 or p + 4 >= n:
        return b[i] if p + 1 == n else avg(b[i], b[i + step])
    v = b[i - 2 * step] + b[i + 3 * step] + 5 * (4 * b[i] - b[i - step] + 4 * b[i + step] - b[i + 2 * step]) + 16
    return clamp(v >> 5, 0, PX_MAX)


def _bicubic(d, s, r0, w, h):
    p1, p2, p3 = r0 + h, r0 + 2 * h, r0 + 3 * h
    for y in range(h):
        for x in range(w):
            d[(p1 + y) * s + x] = _half(d, (r0 + y) * s + x, 1, x, w)
    for y in range(h):
        for x in range(w):
            d[(p2 + y) * s + x] = _half(d, (r0 + y) * s + x, s, y, h)
    for y in range(h):
        for x in range(w):
            d[(p3 + y) * s + x] = _half(d, (p2 + y) * s + x, 1, x, w)


def build_super(o, frame):
    """SuperBuilder::build on one packed I420 frame (portable.rs:94-148): bytes in, bytes out at 8
    bits; a sequence of samples in, a list of samples out at 10 bits."""
    w, h = o.width, o.height
    cw, ch = w // 2, h // 2
    sh = super_plane_height(h, o.pel, o.levels, o.full)
    wide = PX_MAX > 255
    y, u, v = ([0] * (w * sh), [0] * (cw * (sh // 2)), [0] * (cw * (sh // 2))) if wide else \
        (bytearray(w * sh), bytearray(cw * (sh // 2)), bytearray(cw * (sh // 2)))
    f = [int(x) for x in frame] if wide else bytes(frame)
    build_plane(y, w, f[:w * h], w, w, h, w, h, False, o)
    build_plane(u, cw, f[w * h:w * h + cw * ch], cw, cw, ch, w, h, True, o)
    build_plane(v, cw, f[w * h + cw * ch:], cw, cw, ch, w, h, True, o)
    return list(y) + list(u) + list(v) if wide else bytes(y + u + v)


# ------------------------------------------------------------------ analyse_opts.rs
class AnalyseOpts:
    pass


def overlap_from_mode(bw, bh, mode):
    if mode == 0:
        return 0, 0
    if mode == 1:
        return tdiv(bw, 8), tdiv(bh, 8)
    if mode == 2:
        return tdiv(bw, 4), tdiv(bh, 4)
    if mode == 3:
        return tdiv(bw, 2), tdiv(bh, 2)
    raise ValueError("SVAnalyse: overlap must be 0, 1 (=1/8*block), 2 (=1/4*block) or 3 (=1/2*block)")


def auto_search_levels(w, h, bw, bh, ox, oy):
    sx, sy = max(bw - ox, 1), max(bh - oy, 1)
    gw, gh = max(tdiv(w - ox, sx), 0), max(tdiv(h - oy, sy), 0)
    if gw <= 0 or gh <= 0:
        return 1
    ex, ey = ox + sx * gw, oy + sy * gh
    lv = 0
    while True:
        if tdiv((ex >> lv) - ox, sx) <= 0 or tdiv((ey >> lv) - oy, sy) <= 0:
            break
        lv += 1
        if lv > 12:
            break
    return max(lv, 1)


def analyse_from_opt(opt, sdata, src_w=0, src_h=0):
    t = tree_of(opt)
    raw = sdata & U64
    h, w, pel, lv, sel = raw & 0xFFFF, (raw >> 16) & 0xFFFF, (raw >> 32) & 0xFF, (raw >> 40) & 0xFF, (raw >> 48) & 0xFF
    if w <= 0 or h <= 0 or not 1 <= pel <= 4 or lv <= 0:
        raise ValueError("SVAnalyse: invalid super clip params")
    o = AnalyseOpts()
    o.width, o.height, o.pel, o.super_levels, o.selector = w, h, pel, lv, sel
    o.vectors = as_i32(first(int_at(t, ("vectors",)), 3))
    if not 1 <= o.vectors <= 3:
        raise ValueError("SVAnalyse: vectors must be 1, 2 or 3")
    bw = as_i32(first(int_at(t, ("block", "w")), 16))
    bh = as_i32(first(int_at(t, ("block", "h")), bw))
    if bw not in (4, 8, 16, 32):
        raise ValueError("SVAnalyse: block.w must be 4/8/16/32")
    om = as_i32(first(int_at(t, ("block", "overlap")), 2))
    ox, oy = overlap_from_mode(bw, bh, om)
    o.delta = as_i32(first(int_at(t, ("special", "delta")), int_at(t, ("delta",)), 1))
    lam = first(float_at(t, ("main", "penalty", "lambda")), float_at(t, ("penalty", "lambda")), 10.0)
    lsad = as_i32(first(int_at(t, ("main", "penalty", "lsad")), int_at(t, ("penalty", "lsad")), 8000))
    plevel = first(float_at(t, ("main", "penalty", "plevel")), float_at(t, ("penalty", "plevel")), 1.5)
    o.plevel = 0.01 if plevel != plevel else max(plevel, 0.01)
    pi = lambda k, d: as_i32(first(int_at(t, ("main", "penalty", k)), int_at(t, ("penalty", k)), d))
    o.pnew, o.pglobal, o.pzero, o.pnbour, o.prev = pi("pnew", 50), pi("pglobal", 50), pi("pzero", 100), pi("pnbour", 50), pi("prev", 0)
    o.search_type = as_i32(first(int_at(t, ("main", "search", "type")), int_at(t, ("search", "type")), 4))
    o.distance = as_i32(first(int_at(t, ("main", "search", "distance")), int_at(t, ("search", "distance")), 2))
    o.coarse_search_type = as_i32(first(int_at(t, ("main", "search", "coarse", "type")),
                                        int_at(t, ("search", "coarse", "type")), o.search_type))
    o.coarse_distance = as_i32(first(int_at(t, ("main", "search", "coarse", "distance")),
                                     int_at(t, ("search", "coarse", "distance")), 0))
    cbs = as_i32(first(int_at(t, ("main", "search", "coarse", "bad", "sad")),
                       int_at(t, ("search", "coarse", "bad", "sad")), 1000))
    o.coarse_bad_range = as_i32(first(int_at(t, ("main", "search", "coarse", "bad", "range")), -24))
    o.fine_satd = first(bool_at(t, ("main", "search", "satd")), bool_at(t, ("search", "satd")), False)
    o.coarse_satd = first(bool_at(t, ("main", "search", "coarse", "satd")), True)
    r = lookup(t, ("refine",)) if t is not None else None
    ref0 = r[0] if isinstance(r, Arr) and len(r) else None
    th = int_at(ref0, ("thsad",)) if ref0 is not None else None
    o.refine_thsad = None if th is None else tdiv(as_i32(as_i32(th) * max(tdiv(bw, 2) * tdiv(bh, 2), 1)), 32)
    o.refine_search_type = as_i32(first(int_at(ref0, ("search", "type")) if ref0 is not None else None, o.search_type))
    o.refine_distance = as_i32(first(int_at(ref0, ("search", "distance")) if ref0 is not None else None, o.distance))
    o.refine_satd = first(bool_at(ref0, ("search", "satd")) if ref0 is not None else None, o.fine_satd)
    o.sort = first(bool_at(t, ("main", "search", "sort")), bool_at(t, ("sort",)), True)
    levels = max(min(auto_search_levels(w, h, bw, bh, ox, oy), lv), 1)
    ml = int_at(t, ("main", "levels"))
    if ml is not None and ml > 0:
        levels = max(min(as_i32(ml), lv), 1)
    area = float(max(bw * bh, 1))
    o.lambda_ = f64_as_i32(2.0 * area * 1000.0 * 0.015625 * lam)
    scale = tdiv(max(bw * bh, 1), 32)
    o.lsad, o.coarse_bad_sad = sat_i32(lsad * scale), sat_i32(cbs * scale)
    o.block_w, o.block_h, o.overlap_x, o.overlap_y, o.levels = bw, bh, ox, oy, levels
    if src_w > 0:
        o.width = src_w
    if src_h > 0:
        o.height = src_h
    return o


def output_block(o):
    if o.refine_thsad is not None:
        return max(tdiv(o.block_w, 2), 4), max(tdiv(o.block_h, 2), 4), max(tdiv(o.overlap_x, 2), 0), max(tdiv(o.overlap_y, 2), 0)
    return o.block_w, o.block_h, o.overlap_x, o.overlap_y


def grid(o, bw, bh, ox, oy):
    sx, sy = max(bw - ox, 1), max(bh - oy, 1)
    return max(tdiv(o.width - ox, sx), 1), max(tdiv(o.height - oy, sy), 1)


# ------------------------------------------------------------------ analyse_search.rs
class Planes:
    def __init__(self, so, data: bytes):
        w = so.width
        sh = super_plane_height(so.height, so.pel, so.levels, so.full)
        cw = w // 2
        yl, cl = w * sh, cw * (sh // 2)
        self.y, self.u, self.v = data[:yl], data[yl:yl + cl], data[yl + cl:yl + 2 * cl]
        self.ys, self.cs = w, cw
        self.lw, self.lh, self.pel, self.full = w, so.height, so.pel, so.full

    def yoff(self, level):
        y = 0
        for lv in range(level):
            y += reduce_dim(self.lh, lv) * (self.pel * self.pel if lv == 0 and self.full else 1)
        return y

    def coff(self, level):
        y = 0
        for lv in range(level):
            y += max(reduce_dim(self.lh, lv) // 2, 1) * (self.pel * self.pel if lv == 0 and self.full else 1)
        return y

    def size(self, level):
        return reduce_dim(self.lw, level), reduce_dim(self.lh, level)


def had4(d):
    t = []
    for i in range(4):
        r = d[4 * i:4 * i + 4]
        s0, s1, s2, s3 = r[0] + r[1], r[0] - r[1], r[2] + r[3], r[2] - r[3]
        t.append((s0 + s2, s1 + s3, s0 - s2, s1 - s3))
    s = 0
    for j in range(4):
        s0, s1, s2, s3 = t[0][j] + t[1][j], t[0][j] - t[1][j], t[2][j] + t[3][j], t[2][j] - t[3][j]
        s += abs(s0 + s2) + abs(s1 + s3) + abs(s0 - s2) + abs(s1 - s3)
    return max(s, 0)


def mv_bounds(px, py, bw, bh, lw, lh, pel):
    pel = max(pel, 1)
    return -pel * px, -pel * py, pel * (lw - px - bw) + 1, pel * (lh - py - bh) + 1


def edge_shift(px, py, mx, my, bw, bh, lw, lh, pel):
    pel = max(pel, 1)
    a, b, c, d = mv_bounds(px, py, bw, bh, lw, lh, pel)
    ox = mx - a if mx < a else (mx + 1 - c if c > a and mx >= c else 0)
    oy = my - b if my < b else (my + 1 - d if d > b and my >= d else 0)
    if ox == 0 and oy == 0:
        return None
    cx, cy = clamp(px - ox, 0, max(lw - bw, 0)), clamp(py - oy, 0, max(lh - bh, 0))
    if pel == 1:
        return cx, cy, cx + mx, cy + my
    if pel == 4:
        return cx, cy, (4 * cx + mx) >> 2, (4 * cy + my) >> 2
    return cx, cy, (2 * cx + mx) >> 1, (2 * cy + my) >> 1


def satd_block(sbuf, sbase, ss, rbuf, rbase, rs, n):  # satd_interior at flat (wrapped) bases
    tot = 0
    for ty in range(n // 4):
        for tx in range(n // 4):
            d = [get(sbuf, us(sbase + (ty * 4 + r) * ss + tx * 4 + c), 0) - get(rbuf, us(rbase + (ty * 4 + r) * rs + tx * 4 + c), 0)
                 for r in range(4) for c in range(4)]
            tot = sat_u32(tot + had4(d))
    return tot >> 1


def sad_block(sbuf, sbase, ss, rbuf, rbase, rs, w, h):
    return sum(abs(get(sbuf, us(sbase + r * ss + c), 0) - get(rbuf, us(rbase + r * rs + c), 0)) for r in range(h) for c in range(w))


def satd_edge(s, ss, srow, sx0, sy0, r, rs, rrow, rx0, ry0, width, height, n):
    tot = 0
    for ty in range(n // 4):
        for tx in range(n // 4):
            d = []
            for rr in range(4):
                sy = clamp(sy0 + ty * 4 + rr, 0, max(height - 1, 0))
                ry = clamp(ry0 + ty * 4 + rr, 0, max(height - 1, 0))
                for c in range(4):
                    sx = clamp(sx0 + tx * 4 + c, 0, max(width - 1, 0))
                    rx = clamp(rx0 + tx * 4 + c, 0, max(width - 1, 0))
                    d.append(get(s, (srow + sy) * ss + sx, 0) - get(r, (rrow + ry) * rs + rx, 0))
            tot = sat_u32(tot + had4(d))
    return tot >> 1


def cost_edge(S, R, level, px, py, bw, bh, mx, my, satd, pel):  # block_cost_edge_lc
    lw, lh = S.size(level)
    e = edge_shift(px, py, mx, my, bw, bh, lw, lh, pel)
    if e is None:
        return None
    cx, cy, rx0, ry0 = e
    yo = S.yoff(level)
    sub = ((my & 1) * pel + (mx & 1)) if level == 0 and pel >= 2 else 0
    cr0, rr0 = yo, yo + sub * lh
    if satd and bw in (4, 8, 16, 32) and bh in (4, 8, 16, 32) and bw == bh:
        L = satd_edge(S.y, S.ys, cr0, cx, cy, R.y, R.ys, rr0, rx0, ry0, lw, lh, bw)
    else:
        L = 0
        for row in range(bh):
            sy, ry = clamp(cy + row, 0, max(lh - 1, 0)), clamp(ry0 + row, 0, max(lh - 1, 0))
            for col in range(bw):
                sx, rx = clamp(cx + col, 0, max(lw - 1, 0)), clamp(rx0 + col, 0, max(lw - 1, 0))
                L = sat_u32(L + abs(get(S.y, (cr0 + sy) * S.ys + sx, 0) - get(R.y, (rr0 + ry) * R.ys + rx, 0)))
    cw, ch, clw, clh = bw // 2, bh // 2, lw // 2, lh // 2
    ccx, ccy = (px >> 1) - ((px - cx) >> 1), (py >> 1) - ((py - cy) >> 1)
    crx, cry = ((mx >> 1) + 2 * ccx) >> 1, ((my >> 1) + 2 * ccy) >> 1
    co = S.coff(level)
    cref = co + sub * clh
    if satd and cw == ch and cw in (4, 8, 16):
        C = sat_u32(satd_edge(S.u, S.cs, co, ccx, ccy, R.u, R.cs, cref, crx, cry, clw, clh, cw)
                    + satd_edge(S.v, S.cs, co, ccx, ccy, R.v, R.cs, cref, crx, cry, clw, clh, cw))
    else:
        C = 0
        for row in range(ch):
            sy, ry = clamp(ccy + row, 0, max(clh - 1, 0)), clamp(cry + row, 0, max(clh - 1, 0))
            for col in range(cw):
                sx, rx = clamp(ccx + col, 0, max(clw - 1, 0)), clamp(crx + col, 0, max(clw - 1, 0))
                C = sat_u32(C + abs(get(S.u, (co + sy) * S.cs + sx, PX_MID) - get(R.u, (cref + ry) * R.cs + rx, PX_MID)))
                C = sat_u32(C + abs(get(S.v, (co + sy) * S.cs + sx, PX_MID) - get(R.v, (cref + ry) * R.cs + rx, PX_MID)))
    return L, sat_u32(C * 4)


def luma_interior(S, R, level, px, py, bw, bh, mx, my, satd, pel):  # block_cost_luma_interior
    lw, lh = S.size(level)
    px = px - (1 if level > 0 and px + bw >= lw else 0)
    py = py - (1 if level > 0 and py + bh >= lh else 0)
    pxu, pyu = us(px), us(py)
    yo = S.yoff(level)
    if level == 0 and pel >= 2:
        sub, mvx, mvy = (my & 1) * pel + (mx & 1), mx >> 1, my >> 1
    else:
        sub, mvx, mvy = 0, mx, my
    cr0, rr0 = yo, yo + sub * lh
    if satd and bw in (4, 8, 16, 32) and bh in (4, 8, 16, 32) and bw == bh:
        n = bw
        rx0, ry0 = as_i32(pxu) + mvx, as_i32(pyu) + mvy

        def smul(a, b):
            a, b = a & U64, b & U64
            return U64 if a * b > U64 else a * b

        def sadd(a, b):
            return U64 if a + b > U64 else a + b

        send = sadd(smul((cr0 + pyu + n - 1) & U64, S.ys), (pxu + n) & U64)
        rend = sadd(smul((rr0 + ry0 + n - 1) & U64, R.ys), max(rx0, 0) + n) if ry0 >= 0 else U64
        if ((pxu + n) & U64) <= lw and ((pyu + n) & U64) <= lh and rx0 >= 0 and ry0 >= 0 and rx0 + n <= lw \
                and ry0 + n <= lh and send <= len(S.y) and rend <= len(R.y):
            return satd_block(S.y, (cr0 + pyu) * S.ys + pxu, S.ys, R.y, (rr0 + ry0) * R.ys + rx0, R.ys, n)
        tot = 0
        for ty in range(n // 4):
            for tx in range(n // 4):
                d = []
                for r in range(4):
                    sy = (pyu + ty * 4 + r) & U64
                    ry = clamp(py + ty * 4 + r + mvy, 0, lh - 1)
                    for c in range(4):
                        sx = (pxu + tx * 4 + c) & U64
                        rx = clamp(px + tx * 4 + c + mvx, 0, lw - 1)
                        a = get(S.y, (cr0 + sy) * S.ys + sx, 0) if sy < lh and sx < lw else 0
                        d.append(a - get(R.y, (rr0 + ry) * R.ys + rx, 0))
                tot = sat_u32(tot + had4(d))
        return tot >> 1
    rx0, ry0 = px + mvx, py + mvy
    if px >= 0 and py >= 0 and rx0 >= 0 and ry0 >= 0 and px + bw <= lw and py + bh <= lh and rx0 + bw <= lw \
            and ry0 + bh <= lh and bw in (4, 8, 16, 32):
        return sad_block(S.y, (cr0 + pyu) * S.ys + pxu, S.ys, R.y, (rr0 + ry0) * R.ys + rx0, R.ys, bw, bh)
    sad = 0
    for row in range(bh):
        sy = (pyu + row) & U64
        ry = clamp(py + row + mvy, 0, lh - 1)
        if sy >= lh:
            break
        for col in range(bw):
            sx = (pxu + col) & U64
            rx = clamp(px + col + mvx, 0, lw - 1)
            if sx >= lw:
                break
            sad = sat_u32(sad + abs(get(S.y, (cr0 + sy) * S.ys + sx, 0) - get(R.y, (rr0 + ry) * R.ys + rx, 0)))
    return sad


def chroma_x4(S, R, level, pel, mx, my, px, py, bw, bh, lw, lh, satd):  # chroma_sad_x4 (px, py are usize)
    cw, ch = bw // 2, bh // 2
    if cw < 4 or ch < 4:
        return 0
    cpx, cpy, clw, clh = px // 2, py // 2, lw // 2, lh // 2
    co = S.coff(level)
    if level == 0 and pel >= 2:
        sub, mcx, mcy = (my & 1) * pel + (mx & 1), mx >> 2, my >> 2
    else:
        sub, mcx, mcy = 0, mx >> 1, my >> 1
    cref = co + (sub * clh if level == 0 and pel > 1 else 0)
    if cw in (4, 8, 16):
        rx0, ry0 = as_i32(cpx) + mcx, as_i32(cpy) + mcy
        if cpx + cw <= clw and cpy + ch <= clh and rx0 >= 0 and ry0 >= 0 and rx0 + cw <= clw and ry0 + ch <= clh:
            su, ru = (co + cpy) * S.cs + cpx, (cref + ry0) * R.cs + rx0
            e = (ch - 1) * S.cs + cw
            if su + e <= len(S.u) and su + e <= len(S.v) and ru + e <= len(R.u) and ru + e <= len(R.v):
                if satd:
                    a = satd_block(S.u, su, S.cs, R.u, ru, R.cs, cw)
                    b = satd_block(S.v, su, S.cs, R.v, ru, R.cs, cw)
                else:
                    a = sad_block(S.u, su, S.cs, R.u, ru, R.cs, cw, ch)
                    b = sad_block(S.v, su, S.cs, R.v, ru, R.cs, cw, ch)
                return sat_u32(sat_u32(a + b) * 4)
    t = 0
    for row in range(ch):
        sy = cpy + row
        ry = clamp(as_i32(cpy) + row + mcy, 0, clh - 1)
        if sy >= clh:
            break
        for col in range(cw):
            sx = cpx + col
            rx = clamp(as_i32(cpx) + col + mcx, 0, clw - 1)
            if sx >= clw:
                break
            t = sat_u32(t + abs(get(S.u, (co + sy) * S.cs + sx, PX_MID) - get(R.u, (cref + ry) * R.cs + rx, PX_MID)))
            t = sat_u32(t + abs(get(S.v, (co + sy) * S.cs + sx, PX_MID) - get(R.v, (cref + ry) * R.cs + rx, PX_MID)))
    return sat_u32(t * 4)


def cost_lc(S, R, level, px, py, bw, bh, mx, my, satd, pel):  # block_cost_lc -> (luma, chroma)
    pel = max(pel, 1)
    e = cost_edge(S, R, level, px, py, bw, bh, mx, my, satd, pel)
    if e is not None:
        return e
    lw, lh = S.size(level)
    return (luma_interior(S, R, level, px, py, bw, bh, mx, my, satd, pel),
            chroma_x4(S, R, level, pel, mx, my, us(px), us(py), bw, bh, lw, lh, satd))


class Ctx:
    pass


def pen(pnew, x):
    return x + ((pnew * x) >> 8)


def check(c, mv, best, label=None):
    """exact_check / exact_check_dir; best = [mv, sad, cost]; returns True when accepted."""
    a, b, cc, d = c.bounds
    if not (mv[0] >= a and mv[1] >= b and mv[0] < cc and mv[1] < d):
        return False
    motion = (c.lam * ((c.pred[0] - mv[0]) ** 2 + (c.pred[1] - mv[1]) ** 2)) >> 8
    if motion >= best[2]:
        return False
    lw, lh = c.S.size(c.level)
    shifted = edge_shift(c.px, c.py, mv[0], mv[1], c.bw, c.bh, lw, lh, max(c.pel, 1)) is not None
    if shifted or c.pnew < 0:
        L, C = cost_lc(c.S, c.R, c.level, c.px, c.py, c.bw, c.bh, mv[0], mv[1], c.satd, c.pel)
        C = C if c.chroma else 0
        sad, cost = sat_u32(L + C), motion + pen(c.pnew, L) + pen(c.pnew, C)
    else:
        L = luma_interior(c.S, c.R, c.level, c.px, c.py, c.bw, c.bh, mv[0], mv[1], c.satd, max(c.pel, 1))
        lb = motion + pen(c.pnew, L)
        if lb >= best[2]:
            return False
        if not c.chroma:
            sad, cost = L, lb
        else:
            C = chroma_x4(c.S, c.R, c.level, max(c.pel, 1), mv[0], mv[1], us(c.px), us(c.py), c.bw, c.bh, lw, lh, c.satd)
            sad, cost = sat_u32(L + C), lb + pen(c.pnew, C)
    if cost < best[2]:
        if label is None:
            best[0] = mv
        best[1], best[2] = sad, cost
        return True
    return False


HEX2 = [(-1, -2), (-2, 0), (-1, 2), (1, 2), (2, 0), (1, -2), (-1, -2), (-2, 0)]
MOD6M1 = [5, 0, 1, 2, 3, 4, 5, 0]
HEX4 = [(-4, 2), (-4, 1), (-4, 0), (-4, -1), (-4, -2), (4, -2), (4, -1), (4, 0), (4, 1), (4, 2), (2, 3), (0, 4),
        (-2, 3), (-2, -3), (0, -4), (2, -3)]


def expanding(c, center, r, step, best):
    i = -r + step
    while i < r:
        check(c, (center[0] + i, center[1] - r), best)
        check(c, (center[0] + i, center[1] + r), best)
        i += step
    j = -r + step
    while j < r:
        check(c, (center[0] - r, center[1] + j), best)
        check(c, (center[0] + r, center[1] + j), best)
        j += step
    for dx, dy in ((-r, -r), (-r, r), (r, -r), (r, r)):
        check(c, (center[0] + dx, center[1] + dy), best)


def hex2(c, radius, best):
    bx, by = best[0]
    if radius > 1:
        d = -2
        for i in range(6):
            if check(c, (bx + HEX2[i + 1][0], by + HEX2[i + 1][1]), best, label=i):
                d = i
        if d != -2:
            bx += HEX2[d + 1][0]
            by += HEX2[d + 1][1]
            it = 1
            a, b, cc, dd = c.bounds
            while it < tdiv(radius, 2) and a <= bx < cc and b <= by < dd:
                od = MOD6M1[d + 1]
                d = -2
                for k in range(3):
                    if check(c, (bx + HEX2[od + k][0], by + HEX2[od + k][1]), best, label=od + k - 1):
                        d = od + k - 1
                if d == -2:
                    break
                bx += HEX2[d + 1][0]
                by += HEX2[d + 1][1]
                it += 1
        best[0] = (bx, by)
    expanding(c, (bx, by), 1, 1, best)


def umh(c, center, radius, best):
    d = 1
    while d < radius:
        check(c, (center[0] - d, center[1]), best)
        check(c, (center[0] + d, center[1]), best)
        d += 2
    d = 1
    while d < radius:
        check(c, (center[0], center[1] - d), best)
        check(c, (center[0], center[1] + d), best)
        d += 2
    for s in range(1, max(tdiv(radius, 4), 1) + 1):
        for dx, dy in HEX4:
            check(c, (center[0] + dx * s, center[1] + dy * s), best)
    hex2(c, radius, best)


def refine(c, stype, radius, best):
    if stype == 2:
        hex2(c, radius, best)
    elif stype == 3:
        umh(c, best[0], radius, best)
    elif stype == 4:
        cx, cy = best[0]
        for y in range(cy - radius, cy + radius + 1):
            for x in range(cx - radius, cx + radius + 1):
                check(c, (x, y), best)


def exact_sad(S, R, level, px, py, bw, bh, mv, satd, pel, chroma):
    if not chroma:
        e = cost_edge(S, R, level, px, py, bw, bh, mv[0], mv[1], satd, max(pel, 1))
        if e is not None:
            return e[0]
        return luma_interior(S, R, level, px, py, bw, bh, mv[0], mv[1], satd, max(pel, 1))
    L, C = cost_lc(S, R, level, px, py, bw, bh, mv[0], mv[1], satd, pel)
    return sat_u32(L + C)


def level_grid(o, level):
    sx, sy = max(o.block_w - o.overlap_x, 1), max(o.block_h - o.overlap_y, 1)
    gw0, gh0 = max(tdiv(o.width - o.overlap_x, sx), 0), max(tdiv(o.height - o.overlap_y, sy), 0)
    ex, ey = o.overlap_x + sx * gw0, o.overlap_y + sy * gh0
    gw = max(tdiv((ex >> level) - o.overlap_x, sx), 1)
    gh = max(tdiv((ey >> level) - o.overlap_y, sy), 1)
    return gw + (1 if level > 0 else 0), gh + (1 if level > 0 else 0)


def init_order(gw, gh):
    out = []
    for y in range(1, gh - 1):
        xs = range(1, gw - 1) if y % 2 == 0 else range(gw - 2, 0, -1)
        out += [(x, y) for x in xs]
    for x in range(gw):
        out.append((x, 0))
        if gh > 1:
            out.append((x, gh - 1))
    for y in range(1, gh - 1):
        out.append((0, y))
        if gw > 1:
            out.append((gw - 1, y))
    return out


def level_order(gw, gh, level):
    e = 1 if level > 0 else 0
    bw, bh = gw - e, gh - e
    o = init_order(bw, bh)
    if e:
        o += [(x, bh) for x in range(bw + 1)] + [(bw, y) for y in range(bh)]
    return o


def refine_order(coarse, cgw, cgh, gw, gh, level):
    if level == 0:
        return init_order(gw, gh)
    sw, sh, dw, dh = cgw - 1, cgh - 1, gw - 1, gh - 1
    ex, ey = max(dw - 2 * sw, 0), max(dh - 2 * sh, 0)
    inner, bound, seen = [], [], set()

    def add(x, y):
        if x < 0 or y < 0 or x >= dw or y >= dh or (x, y) in seen:
            return
        seen.add((x, y))
        (inner if 0 < x < dw - 1 and 0 < y < dh - 1 else bound).append((x, y))

    for x, y in coarse:
        if x >= sw or y >= sh:
            continue
        l, t = 2 * x, 2 * y
        for dx, dy in ((0, 0), (1, 0), (1, 1), (0, 1)):
            add(l + dx, t + dy)
        if x == sw - 1:
            for dx in range(2, 2 + ex):
                for dy in range(0, 2 + (ey if y == sh - 1 else 0)):
                    add(l + dx, t + dy)
        if y == sh - 1:
            for dy in range(2, 2 + ey):
                for dx in range(2):
                    add(l + dx, t + dy)
    return inner + bound + [(x, dh) for x in range(dw + 1)] + [(dw, y) for y in range(dh)]


def reorder(order, field, gw, gh, bw, bh):
    count = (gw - 1) * (gh - 1)
    shift = max(tdiv(bw * bh, 8), 1).bit_length() - 1 + 1
    base = [(x, y) for y in range(gh - 1) for x in range(gw - 1)]
    base.sort(key=lambda p: field[p[1] * gw + p[0]][2] >> shift)  # stable
    order[:count] = base


def interpolate(coarse, cgw, cgh, gw, gh, bw, bh, ox, oy, pel):
    out = [[0, 0, 0, 0] for _ in range(gw * gh)]
    proj = [[0, 0, U32, 0] for _ in range(gw * gh)]
    cw, ch = cgw - 1, cgh - 1
    for y in range(gh - 1):
        for x in range(gw - 1):
            if x < 2 * cw and y < 2 * ch:
                p = coarse[(y >> 1) * cgw + (x >> 1)]
            else:
                e = ch + min(x >> 1, cw) - min(y >> 1, ch)
                ex, ey = (e, ch) if e <= cw else (cw, cw + ch - e)
                p = coarse[ey * cgw + ex]
            vx, vy = p[0] * 2 * pel, p[1] * 2 * pel
            v = [clamp(vx, -32768, 32767), clamp(vy, -32768, 32767), p[2], p[3]]
            out[y * gw + x] = v
            if x >= 2 * cw or y >= 2 * ch:
                continue
            tx = clamp(tdiv(vx + (bw >> 1) + (bw - ox) * x, bw - ox), 0, gw - 1)
            ty = clamp(tdiv(vy + (bh >> 1) + (bh - oy) * y, bh - oy), 0, gh - 1)
            if v[2] < proj[ty * gw + tx][2]:
                proj[ty * gw + tx] = [i16(-v[0]), i16(-v[1]), v[2], 0]
    return out, proj


def global_doubled(field):
    def mode(vals):
        vals = sorted(vals)
        best, bc, i = (vals[0] if vals else 0), 0, 0
        while i < len(vals):
            j = i + 1
            while j < len(vals) and vals[j] == vals[i]:
                j += 1
            if j - i > bc:
                best, bc = vals[i], j - i
            i = j
        return best

    mx, my = mode([v[0] for v in field]), mode([v[1] for v in field])
    sx = sy = n = 0
    for v in field:
        if abs(v[0] - mx) < 6 and abs(v[1] - my) < 6:
            sx += v[0]
            sy += v[1]
            n += 1
    if n == 0:
        return 2 * mx, 2 * my
    sg = lambda s: (s > 0) - (s < 0)
    return 2 * tdiv(sx + tdiv(sg(sx) * n, 2), n), 2 * tdiv(sy + tdiv(sg(sy) * n, 2), n)


def powi(a, b):
    r = 1.0
    while True:
        if b & 1:
            r *= a
        b = tdiv(b, 2)
        if b == 0:
            break
        a *= a
    return r


def luma_dc(S, level, px, py, bw, bh):
    lw, lh = S.size(level)
    yo = S.yoff(level)
    s = n = 0
    for row in range(bh):
        y = (us(py) + row) & U64
        if y >= lh:
            break
        for col in range(bw):
            x = (us(px) + col) & U64
            if x >= lw:
                break
            s += get(S.y, (yo + y) * S.ys + x, 0)
            n += 1
    return 0 if n == 0 else min((s // n) >> DC_SHIFT, 255)


def plane_activity(data, stride, row, x, width, height, satd):  # :1517-1553
    area = width * height
    vals = [[data[(row + y) * stride + x + i] for i in range(width)] for y in range(height)]
    mean = (sum(map(sum, vals)) & U32) // area
    if not satd:
        return (sum(abs(v - mean) for r in vals for v in r) & U32) // area
    total = 0
    for y in range(0, height, 4):
        for x0 in range(0, width, 4):
            d = [data[(row + y + dy) * stride + x + x0 + dx] - mean for dy in range(4) for dx in range(4)]
            total += had4(d)
    return ((total & U32) >> 1) // area


def block_activity(S, level, px, py, bw, bh, satd):  # :1486-1515
    lw, lh = S.size(level)
    x = px - (1 if level > 0 and px + bw >= lw else 0)
    y = py - (1 if level > 0 and py + bh >= lh else 0)
    luma = plane_activity(S.y, S.ys, S.yoff(level) + y, x, bw, bh, satd)
    cw, ch = tdiv(bw, 2), tdiv(bh, 2)
    u = plane_activity(S.u, S.cs, S.coff(level) + tdiv(py, 2), tdiv(px, 2), cw, ch, satd)
    v = plane_activity(S.v, S.cs, S.coff(level) + tdiv(py, 2), tdiv(px, 2), cw, ch, satd)
    return (luma + u + v) & U32


def adaptive_radius(radius, activity):  # :1478-1484
    if activity < 2:
        return 0
    return ((radius * min(((255 * activity) & U32) // 150, 255)) >> 8) + 1


def search_level(S, R, o, level, glob, prev, field, gw, gh, order):
    bw0, bh0 = o.block_w, o.block_h
    stx, sty = max(bw0 - o.overlap_x, 1), max(bh0 - o.overlap_y, 1)
    pel = max(o.pel, 1) if level == 0 else 1
    nl = max(o.levels, 1)
    d = o.distance if level == 0 else o.coarse_distance
    base_r = (0 if level == 0 and nl > 1 else 10) if d == 0 else abs(d)
    stype = o.search_type if level == 0 else o.coarse_search_type
    satd = o.fine_satd if level == 0 else o.coarse_satd
    bad = 0
    done = set()
    lw, lh = S.size(level)
    for bx, by in order:
        idx = by * gw + bx
        px = lw - bw0 if level > 0 and bx == gw - 1 else bx * stx
        py = lh - bh0 if level > 0 and by == gh - 1 else by * sty
        small = level == o.levels - 1
        bw, bh = (bw0 >> 1, bh0 >> 1) if small else (bw0, bh0)
        if small:
            px, py = px + (bw0 >> 2), py + (bh0 >> 2)
        edge = level > 0 and (bx == gw - 1 or by == gh - 1)
        sx, sy = min(bx, gw - 2), min(by, gh - 2)
        if sy * gw + sx < 0:
            raise RuntimeError("reference panics")
        ip = list(field[sy * gw + sx])
        if edge and not small:
            ip[2] = exact_sad(S, R, level, sx * stx, sy * sty, bw, bh, (ip[0], ip[1]), satd, pel, True)
        elif not edge:
            ip = list(field[idx])
        pred = (ip[0], ip[1])
        lam0 = 0 if small else f64_as_i32(float(o.lambda_) / powi(o.plevel, o.levels - level - 1) / float(max(pel * pel, 1)))
        ls = float(max(tdiv(o.lsad, 3) if small else o.lsad, 1))
        half = -1.0 if ip[2] == U32 else float(ip[2] >> 1)
        try:
            tt = ls / (ls + half)
            lv = float(lam0) * tt * tt
        except ZeroDivisionError:
            lv = float("nan")
        lam = f64_as_i32(21474836.47 if lv != lv else min(lv, 21474836.47))
        radius = base_r
        if level > 0 and o.coarse_distance < 0:
            radius = adaptive_radius(base_r, block_activity(S, level, px, py, bw, bh, satd))
        seeds = [(field[ny * gw + nx][0], field[ny * gw + nx][1])
                 for ny in range(max(by - 1, 0), min(by + 1, gh - 1) + 1)
                 for nx in range(max(bx - 1, 0), min(bx + 1, gw - 1) + 1) if (nx, ny) in done]
        if len(seeds) > 8:
            raise RuntimeError("reference panics")
        c = Ctx()
        c.S, c.R, c.level, c.px, c.py, c.bw, c.bh, c.pel, c.satd, c.chroma = S, R, level, px, py, bw, bh, pel, satd, not small
        c.bounds, c.lam, c.pnew = mv_bounds(px, py, bw, bh, lw, lh, pel), lam, o.pnew

        def special(mv, pn):
            s_ = exact_sad(S, R, level, px, py, bw, bh, mv, satd, pel, not small)
            return [mv, s_, s_ + ((pn * s_) >> 8)]

        fv = ip[2] != U32
        fb = special(pred, 0) if fv else None
        if level == 0 and o.distance == 0:
            best = fb if fv else special((0, 0), 0)
        else:
            pv = prev[idx] if prev is not None and prev[idx][2] != U32 and prev[idx][2] > 0 else None
            pb = special((pv[0], pv[1]), o.prev) if pv else None
            zb, gb = special((0, 0), o.pzero), special(tuple(glob), o.pglobal)
            best = list(fb) if fv else [(0, 0), U32, I64MAX]
            p2 = pred
            if pb and pb[2] < best[2]:
                best, p2 = list(pb), pb[0]
            for cand in (gb, zb):
                if cand[2] < best[2]:
                    best = list(cand)
            for mv in seeds:
                s_ = exact_sad(S, R, level, px, py, bw, bh, mv, satd, pel, not small)
                co = s_ + ((o.pnbour * s_) >> 8)
                if co < best[2]:
                    best = [mv, s_, co]
            best[2] = best[1]
            c.pred = p2
            refine(c, 0 if edge and level == 1 else stype, radius, best)
            found = best[1]
            lim = sat_i32(o.coarse_bad_sad + tdiv(sat_i32(o.coarse_bad_sad * bad), 16))
            if level > 0 and idx > 1 and o.coarse_bad_sad > 0 and as_i32(best[1]) > lim:
                bad += 1
                c.pred = pred
                if o.coarse_bad_range < 0:
                    r = pel
                    while r < -o.coarse_bad_range * pel:
                        expanding(c, (0, 0), r, pel, best)
                        if best[1] < found // 4:
                            break
                        r += pel
                elif o.coarse_bad_range > 0:
                    umh(c, (0, 0), o.coarse_bad_range * pel, best)
                expanding(c, best[0], 1, 1, best)
        field[idx] = [i16(best[0][0]), i16(best[0][1]), sat_u32(best[1] * (3 if small else 1)),
                      luma_dc(S, level, px, py, bw, bh)]
        done.add((bx, by))


def rescale(field, w, h, blk):
    diag = max(f64_as_i32(math.sqrt(float(w) * float(w) + float(h) * float(h))), 0)
    den = max(sat_i32(diag * max(blk, 1)), 1)
    for v in field:
        ratio = tdiv(100 * (abs(v[0]) + abs(v[1])), den)
        sc = as_i32(v[2])
        if ratio >= 51:
            sc = sat_i32(sc * 20)
        elif ratio >= 16:
            w71 = as_i32((((3926827243 * (sc & U32)) & U64) * ((ratio - 15) & U32) & U64) >> 32)
            sc = sat_i32(sc + 9 * ((w71 >> 31) + (w71 >> 5)))
        v[2] = (sc & U32) & 0xFFFFFF


def exact_clip(mv, bounds):  # :1269-1273
    a, b, c, d = bounds
    return min(max(mv[0], a), max(c - 1, a)), min(max(mv[1], b), max(d - 1, b))


def recalculate(S, R, o, field, ogw, ogh):
    """exact_recalculate (:1326-1451): the level-0 field resampled onto blocks of half the size,
    each re-searched from its bilinear-interpolated parent vector when the parent's score is high."""
    if o.refine_thsad is None:
        return field
    obw, obh, oox, ooy = o.block_w, o.block_h, o.overlap_x, o.overlap_y
    bw, bh, ox, oy = output_block(o)
    gw, gh = grid(o, bw, bh, ox, oy)
    osx, osy = max(obw - oox, 1), max(obh - ooy, 1)
    sx, sy = max(bw - ox, 1), max(bh - oy, 1)
    pel = max(o.pel, 1)
    lw, lh = S.size(0)
    out = [None] * (gw * gh)

    def get(x, y):
        return field[min(max(y, 0), ogh - 1) * ogw + min(max(x, 0), ogw - 1)]

    for by in range(gh):
        backwards = o.sort and by & 1
        for pos in range(gw):
            bx = gw - 1 - pos if backwards else pos
            cx, cy = tdiv(bw, 2) + sx * bx, tdiv(bh, 2) + sy * by
            px0, py0 = tdiv(cx - tdiv(obw, 2), osx), tdiv(cy - tdiv(obh, 2), osy)
            dxw = max(cx - (tdiv(obw, 2) + osx * px0), 0)
            dyw = max(cy - (tdiv(obh, 2) + osy * py0), 0)
            corners = (get(px0, py0), get(px0 + 1, py0), get(px0, py0 + 1), get(px0 + 1, py0 + 1))

            def bilinear(k):  # i64 with div_euclid (floor, the divisors are positive)
                a, b, c, d = (v[k] for v in corners)
                top = a * osx + dxw * (b - a)
                bottom = c * osx + dxw * (d - c)
                return (top + (dyw * (bottom - top)) // osy) // osx

            mv = (as_i32(bilinear(0)), as_i32(bilinear(1)))
            parent = tdiv(bilinear(2) * (bw * bh), obw * obh)  # i64 `/` truncates
            border = bx == 0 or by == 0 or bx == gw - 1 or by == gh - 1
            factor = 3 if border and bw > 4 else 1
            ebw, ebh = (tdiv(bw, 2), tdiv(bh, 2)) if factor == 3 else (bw, bh)
            epx = bx * sx + (tdiv(bw, 4) if factor == 3 else 0)
            epy = by * sy + (tdiv(bh, 4) if factor == 3 else 0)
            bounds = mv_bounds(epx, epy, ebw, ebh, lw, lh, pel)
            pred = exact_clip(mv, bounds)
            best = [pred, min(max(parent, 0), U32), max(parent, 0)]
            if parent > tdiv(o.refine_thsad, factor):
                sad = exact_sad(S, R, 0, epx, epy, ebw, ebh, pred, o.refine_satd, pel, True)
                best = [pred, sad, sad]
                c = Ctx()
                c.S, c.R, c.level, c.px, c.py, c.bw, c.bh, c.pel = S, R, 0, epx, epy, ebw, ebh, pel
                c.satd, c.chroma, c.pred, c.bounds = o.refine_satd, True, pred, bounds
                c.lam = 0 if by == 0 else tdiv(o.lambda_ >> 2, factor)
                c.pnew = tdiv(o.pnew, factor)
                refine(c, o.refine_search_type, abs(o.refine_distance), best)
            out[by * gw + bx] = [i16(best[0][0]), i16(best[0][1]), sat_u32(best[1] * factor),
                                 luma_dc(S, 0, epx, epy, ebw, ebh)]
    return out


def analyse_pair(cur: Planes, ref: Planes, o):
    dirs = [d for d, bit in ((0, 2), (1, 1)) if o.vectors & bit]
    bidir = len(dirs) == 2
    st = {d: dict(field=None, order=[], glob=(0, 0), proj=None) for d in dirs}
    fgw = fgh = 0
    for level in range(max(o.levels, 1) - 1, -1, -1):
        gw, gh = level_grid(o, level)
        pel = max(o.pel, 1) if level == 0 else 1
        for d in dirs:
            s = st[d]
            s["order"] = level_order(gw, gh, level) if not s["order"] else refine_order(s["order"], fgw, fgh, gw, gh, level)
            if s["field"] is None:
                s["next"], s["proj"] = [[0, 0, 0, 0] for _ in range(gw * gh)], None
            else:
                s["next"], s["proj"] = interpolate(s["field"], fgw, fgh, gw, gh, o.block_w, o.block_h, o.overlap_x, o.overlap_y, pel)
        for d in dirs:
            a, b = (cur, ref) if d == 0 else (ref, cur)
            prev = st[1 - d]["proj"] if bidir else st[d]["proj"]
            search_level(a, b, o, level, st[d]["glob"], prev, st[d]["next"], gw, gh, st[d]["order"])
        for d in dirs:
            s = st[d]
            if level > 0:
                s["glob"] = global_doubled(s["next"])
                reorder(s["order"], s["next"], gw, gh, o.block_w, o.block_h)
            s["field"] = s["next"]
        fgw, fgh = gw, gh
    for d in dirs:
        a, b = (cur, ref) if d == 0 else (ref, cur)
        st[d]["field"] = recalculate(a, b, o, st[d]["field"], fgw, fgh)
    bw = output_block(o)[0]
    for d in dirs:
        rescale(st[d]["field"], o.width, o.height, bw)
    return (st[1]["field"] if 1 in dirs else None), (st[0]["field"] if 0 in dirs else None)


def pack(o, prev, cur) -> bytes:
    bw, bh, ox, oy = output_block(o)
    gw, gh = grid(o, bw, bh, ox, oy)
    n = gw * gh
    flags = (1 if prev is not None else 0) | (2 if cur is not None else 0)
    hdr = [16, 0xA0, flags, bw, bh, o.pel, 1 if o.refine_thsad is not None else o.levels, 0, o.width, o.height,
           ox, oy, gw, gh, o.selector, o.delta]
    out = bytearray(struct.pack("<16i", *hdr))
    for reg in (prev, cur):
        if reg is None:
            continue
        out += struct.pack("<i", 2 * n + 1)
        for v in reg[:n]:
            out += struct.pack("<II", ((v[0] & U32) << 16 & U32) | (v[1] & 0xFFFF), (v[2] & 0xFFFFFF) | (v[3] << 24))
    return bytes(out)


def analyse(so, opt, cur_super: bytes, ref_super: bytes, src_w=0, src_h=0) -> bytes:
    o = analyse_from_opt(opt, pack_data(so), src_w, src_h)
    conv = (lambda a: [int(x) for x in a]) if PX_MAX > 255 else bytes
    bwd, fwd = analyse_pair(Planes(so, conv(cur_super)), Planes(so, conv(ref_super)), o)
    return pack(o, bwd, fwd)
