"""SmoothFps's single-warp frame render (renderer.rs render_mode1_or_2, with and without masks).

CPU: the oracle's C restatement against properties of the render (identity, whole-plane shifts,
super-clip sub-planes) and against a second, independent restatement in Python written from the
reference's scalar loop (small frames). GPU: svpf_render_warp_device through the C ABI against the
oracle, bit-exact, over frame and block sizes, thresholds, both modes, interpolation on and off,
plain and super-clip sources, and after the whole device chain (Super, Analyse, vector planes).
"""
import math

import numpy as np
import pytest

from oracle import oracle as orc

CPU_MAP = [0, 1, 2, 2, -1, 3, 3, 3, -1, -1, -1, 4, -1, 4, -1, 4, -1, -1, -1, -1, -1, -1, -1, -1, 5, -1, -1, -1, 5,
           -1, -1, 5]


def _cfg(w, h, bw, bh, gw, gh, step=1, ox=None, oy=None):
    return dict(width=w, height=h, block_w=bw, block_h=bh, origin_x=bw // 2 if ox is None else ox,
                origin_y=bh // 2 if oy is None else oy, grid_w=gw, grid_h=gh, chroma_y_div=2, source_step=step)


def _grid(w, h, bw, bh):
    """The motion grid of a vector field of bw x bh blocks at half-block steps (extended_grid)."""
    sx, sy = bw // 2, bh // 2
    gw, gh = max((w - bw) // sx + 1, 1), max((h - bh) // sy + 1, 1)
    return gw + ((bw - sx) * gw + sx < w), gh + ((bh - sy) * gh + sy < h)


# ---------------------------------------------------------------- a second restatement (Python)
def _py_render(cfg, chroma, interp, lut, src, stride, span, shift, mx, my, mask=None):
    """render_selected_warp_rows, scalar loop (renderer.rs:876-984), in plain Python."""
    cmap = lambda v: CPU_MAP[v - 1] if 1 <= v <= 32 else -1
    cd = cfg["chroma_y_div"]
    zero = not interp
    if chroma:
        W, H, BW, BH = cfg["width"] // 2, cfg["height"] // cd, cfg["block_w"] // 2, cfg["block_h"] // cd
        ox, oy = (0, 0) if zero else (cfg["origin_x"] // 2, cfg["origin_y"] // cd)
        xs_, ys_ = cmap(cfg["block_w"] // 2), cmap(cfg["block_h"] // 2)
        xd, yd = 2, cd
    else:
        W, H, BW, BH = cfg["width"], cfg["height"], cfg["block_w"], cfg["block_h"]
        ox, oy = (0, 0) if zero else (cfg["origin_x"], cfg["origin_y"])
        xs_, ys_ = cmap(BW), cmap(BH)
        xd, yd = 1, 1
    step = cfg["source_step"]
    maxx, maxy = max(W * step - 1, 0), max(H * step - 1, 0)

    def weights(total, sh):
        out = [(0, 0)] * 32
        scale = 1 << max(sh, 0)
        for p in range(min(total, 32)):
            if sh < 0:
                out[p] = (total - p, p)
            else:
                c = lambda v: int(math.ceil(v * scale / total - 0.5))
                out[p] = (c(total - p), c(p))
        return out

    xw, yw = weights(BW, xs_), weights(BH, ys_)
    mox, moy = (cfg["origin_x"] // 2, cfg["origin_y"] // cd) if chroma else (cfg["origin_x"], cfg["origin_y"])

    def mask_at(x, y):
        i = y * cfg["grid_w"] + x
        return int(mask[i]) if x >= 0 and y >= 0 and i < len(mask) else 0

    def alpha_abs(x, y):  # alpha_at_absolute with the plane's own origin
        ix0 = ix1 = iy0 = iy1 = 0
        if mox <= x:
            ix0 = (x - mox) // BW
            ix1 = ix0 + 1
        if moy <= y:
            iy0 = (y - moy) // BH
            iy1 = iy0 + 1
        fx = (x - mox) % BW if mox < x else 0
        fy = (y - moy) % BH if moy < y else 0
        top = ((BW - fx) * mask_at(ix0, iy0) + fx * mask_at(ix1, iy0)) // BW
        bot = ((BW - fx) * mask_at(ix0, iy1) + fx * mask_at(ix1, iy1)) // BW
        return min(max(((BH - fy) * top + fy * bot) // BH, 0), 255)

    def ip(a, b, total, sh, w):
        s = w[0] * a + w[1] * b
        return int(s / total) if sh < 0 else s >> sh

    def mv(plane, i):
        k = int(plane[i]) if i < len(plane) else 1024
        return int(lut[min(k, 2047)])

    def index(x, y):
        if shift == 0:
            return y * stride + x
        m = (1 << shift) - 1
        return (((y & m) << shift) | (x & m)) * span + (y >> shift) * stride + (x >> shift)

    covers = (shift == 0 or (1 << shift) == step) and index(maxx, maxy) < len(src)
    gw, gh = cfg["grid_w"], cfg["grid_h"]
    dst = np.zeros((H, W), dtype=np.uint8)
    tdiv = lambda a, b: int(a / b)
    for gy in range(-1, gh):
        by = 0 if gy < 0 else oy + BH * gy
        th = oy if gy < 0 else BH
        if by + BH >= H or gy == gh - 1:
            th = H - by
        th = min(by + th, H) - max(by, 0)
        if th <= 0:
            continue
        for gx in range(-1, gw):
            bx = 0 if gx < 0 else ox + BW * gx
            tw = ox if gx < 0 else BW
            if bx + BW >= W or gx == gw - 1:
                tw = W - bx
            if tw <= 0:
                continue
            i00 = max(gy, 0) * gw + max(gx, 0)
            nx = 1 if (gx >= 0 and gx != gw - 1) else 0
            ny = gw if (gy >= 0 and gy != gh - 1) else 0
            idx = [i00, i00 + nx, i00 + ny, i00 + ny + nx]
            sx = [tdiv(mv(mx, i), xd) for i in idx]
            sy = [tdiv(mv(my, i), yd) for i in idx]
            if not interp:
                sx, sy = [sx[0]] * 4, [sy[0]] * 4
            direct = covers and bx * step + min(sx) >= 0 and by * step + min(sy) >= 0 and \
                (bx + tw - 1) * step + max(sx) <= maxx and (by + th - 1) * step + max(sy) <= maxy
            for y in range(th):
                wy = yw[min(y, 31)]
                rx = [ip(sx[0], sx[2], BH, ys_, wy), ip(sx[1], sx[3], BH, ys_, wy)] if interp else [sx[0]] * 2
                ry = [ip(sy[0], sy[2], BH, ys_, wy), ip(sy[1], sy[3], BH, ys_, wy)] if interp else [sy[0]] * 2
                if mask is not None:
                    mk = [int(mask[i]) if i < len(mask) else 0 for i in idx]
                    mrow = [ip(mk[0], mk[2], BH, ys_, wy), ip(mk[1], mk[3], BH, ys_, wy)] if interp else [mk[0]] * 2
                for x in range(tw):
                    wx = xw[min(x, 31)]
                    dx = ip(rx[0], rx[1], BW, xs_, wx) if interp else rx[0]
                    dy = ip(ry[0], ry[1], BW, xs_, wx) if interp else ry[0]
                    X, Y = (bx + x) * step + dx, (by + y) * step + dy
                    if not direct:
                        X, Y = min(max(X, 0), maxx), min(max(Y, 0), maxy)
                    i = index(X, Y)
                    v = int(src[i]) if i < len(src) else 0
                    if mask is not None:
                        bi = index((bx + x) * step, (by + y) * step)
                        base = int(src[bi]) if bi < len(src) else 0
                        a = min(max(ip(mrow[0], mrow[1], BW, xs_, wx), 0), 255) if interp else alpha_abs(bx + x, by + y)
                        v = min(max((v * (255 - a) + base * a + 255) >> 8, 0), 255)
                    dst[by + y, bx + x] = v
    return dst


def _py_dual(cfg, chroma, interp, zero, mode, thr, srcs, strides, spans, shift, mot0, mot1, masks=None, final=None,
             tlimit=0):
    """render_dual_warp_rows + mode11_or_13_pixel / mode21_or_22_pixel (renderer.rs:1031-1172,
    :2918-2943, :615-641) in plain Python."""
    mask = np.maximum(*masks) if masks is not None and mode in (11, 13) else None
    cmap = lambda v: CPU_MAP[v - 1] if 1 <= v <= 32 else -1
    cd = cfg["chroma_y_div"]
    if chroma:
        W, H, BW, BH = cfg["width"] // 2, cfg["height"] // cd, cfg["block_w"] // 2, cfg["block_h"] // cd
        mox, moy = cfg["origin_x"] // 2, cfg["origin_y"] // cd
        xs_, ys_, xd, yd = cmap(cfg["block_w"] // 2), cmap(cfg["block_h"] // 2), 2, cd
    else:
        W, H, BW, BH = cfg["width"], cfg["height"], cfg["block_w"], cfg["block_h"]
        mox, moy = cfg["origin_x"], cfg["origin_y"]
        xs_, ys_, xd, yd = cmap(BW), cmap(BH), 1, 1
    ox, oy = (0, 0) if zero else (mox, moy)
    step = cfg["source_step"]
    maxx, maxy = max(W * step - 1, 0), max(H * step - 1, 0)

    def weights(total, sh):
        out = [(0, 0)] * 32
        for p in range(min(total, 32)):
            c = lambda v: int(math.ceil(v * (1 << max(sh, 0)) / total - 0.5))
            out[p] = (total - p, p) if sh < 0 else (c(total - p), c(p))
        return out

    xw, yw = weights(BW, xs_), weights(BH, ys_)
    ip = lambda a, b, total, sh, w: int((w[0] * a + w[1] * b) / total) if sh < 0 else (w[0] * a + w[1] * b) >> sh
    inv, tl = orc.render_luts(thr)
    luts = [tl, inv]
    gw, gh = cfg["grid_w"], cfg["grid_h"]
    byte = lambda v: min(max(v, 0), 255)
    b256 = lambda a, b, w: byte((a * (256 - w) + b * w) >> 8)

    def index(k, x, y):
        if shift == 0:
            return y * strides[k] + x
        m = (1 << shift) - 1
        return (((y & m) << shift) | (x & m)) * spans[k] + (y >> shift) * strides[k] + (x >> shift)

    def alpha_abs(x, y, mk=None):
        mk = mask if mk is None else mk

        def mat(x, y):
            i = y * gw + x
            return int(mk[i]) if x >= 0 and y >= 0 and i < len(mk) else 0

        ix0 = ix1 = iy0 = iy1 = 0
        if mox <= x:
            ix0 = (x - mox) // BW
            ix1 = ix0 + 1
        if moy <= y:
            iy0 = (y - moy) // BH
            iy1 = iy0 + 1
        fx = (x - mox) % BW if mox < x else 0
        fy = (y - moy) % BH if moy < y else 0
        top = ((BW - fx) * mat(ix0, iy0) + fx * mat(ix1, iy0)) // BW
        bot = ((BW - fx) * mat(ix0, iy1) + fx * mat(ix1, iy1)) // BW
        return byte(((BH - fy) * top + fy * bot) // BH)

    covers = all((shift == 0 or (1 << shift) == step) and index(k, maxx, maxy) < len(srcs[k]) for k in range(2))
    dst = np.zeros((H, W), dtype=np.uint8)
    for gy in range(-1, gh):
        by = 0 if gy < 0 else oy + BH * gy
        th = oy if gy < 0 else BH
        if by + BH >= H or gy == gh - 1:
            th = H - by
        th = min(by + th, H) - max(by, 0)
        if th <= 0:
            continue
        for gx in range(-1, gw):
            bx = 0 if gx < 0 else ox + BW * gx
            tw = ox if gx < 0 else BW
            if bx + BW >= W or gx == gw - 1:
                tw = W - bx
            if tw <= 0:
                continue
            i00 = max(gy, 0) * gw + max(gx, 0)
            nx = 1 if (gx >= 0 and gx != gw - 1) else 0
            ny = gw if (gy >= 0 and gy != gh - 1) else 0
            idx = [i00, i00 + nx, i00 + ny, i00 + ny + nx] if interp else [i00] * 4
            S = []
            for k, (mx, my) in enumerate((mot0, mot1)):
                mv = lambda pl, i: int(luts[k][min(int(pl[i]) if i < len(pl) else 1024, 2047)])
                S.append(([int(mv(mx, i) / xd) for i in idx], [int(mv(my, i) / yd) for i in idx]))
            allx = S[0][0] + S[1][0]
            ally = S[0][1] + S[1][1]
            direct = covers and bx * step + min(allx) >= 0 and by * step + min(ally) >= 0 and \
                (bx + tw - 1) * step + max(allx) <= maxx and (by + th - 1) * step + max(ally) <= maxy
            for y in range(th):
                wy = yw[min(y, 31)]
                rows = []
                for sx, sy in S:
                    rows.append(([ip(sx[0], sx[2], BH, ys_, wy), ip(sx[1], sx[3], BH, ys_, wy)],
                                 [ip(sy[0], sy[2], BH, ys_, wy), ip(sy[1], sy[3], BH, ys_, wy)]) if interp
                                else ([sx[0]] * 2, [sy[0]] * 2))
                if mask is not None:
                    mk = [int(mask[i]) if i < len(mask) else 0 for i in [i00, i00 + nx, i00 + ny, i00 + ny + nx]]
                    mrow = [ip(mk[0], mk[2], BH, ys_, wy), ip(mk[1], mk[3], BH, ys_, wy)] if interp else [mk[0]] * 2
                for x in range(tw):
                    wx = xw[min(x, 31)]
                    vals, curs = [], []
                    for k in range(2):
                        rx, ry = rows[k]
                        dx = ip(rx[0], rx[1], BW, xs_, wx) if interp else rx[0]
                        dy = ip(ry[0], ry[1], BW, xs_, wx) if interp else ry[0]
                        X, Y = (bx + x) * step + dx, (by + y) * step + dy
                        BX, BY = (bx + x) * step, (by + y) * step
                        if not direct:
                            X, Y = min(max(X, 0), maxx), min(max(Y, 0), maxy)
                            BX, BY = min(BX, maxx), min(BY, maxy)
                        i, bi = index(k, X, Y), index(k, BX, BY)
                        vals.append(int(srcs[k][i]) if i < len(srcs[k]) else 0)
                        curs.append(int(srcs[k][bi]) if bi < len(srcs[k]) else 0)
                    def alpha_of(mk):  # alpha_at_absolute, or alpha_at_row over the tile's corners
                        if zero:
                            return alpha_abs(bx + x, by + y, mk)
                        c4 = [int(mk[i]) if i < len(mk) else 0 for i in [i00, i00 + nx, i00 + ny, i00 + ny + nx]]
                        if not interp:
                            return byte(c4[0])
                        r = [ip(c4[0], c4[2], BH, ys_, wy), ip(c4[1], c4[3], BH, ys_, wy)]
                        return byte(ip(r[0], r[1], BW, xs_, wx))

                    b255 = lambda a, b, w: byte((a * (255 - w) + b * w + 255) >> 8)
                    if mode in (21, 22):
                        a0, a1 = alpha_of(masks[0]), alpha_of(masks[1])
                        ea, eb = b255(vals[0], vals[1], a0), b255(vals[1], vals[0], a1)
                        if mode == 21:
                            m = b256(ea, eb, thr)
                        else:
                            m = min(max(b256(curs[0], curs[1], thr), min(ea, eb)), max(ea, eb))
                        if final is not None:
                            m = b255(m, b256(curs[0], curs[1], tlimit), alpha_of(final))
                        dst[by + y, bx + x] = m
                        continue
                    if mode == 13:
                        m = min(max(b256(curs[0], curs[1], thr), min(vals)), max(vals))
                    else:
                        m = b256(vals[0], vals[1], thr)
                    if mask is not None:
                        if zero:
                            a = alpha_abs(bx + x, by + y)
                        else:
                            a = byte(ip(mrow[0], mrow[1], BW, xs_, wx) if interp else mrow[0])
                        m = byte((m * (255 - a) + b256(curs[0], curs[1], thr) * a + 255) >> 8)
                    dst[by + y, bx + x] = m
    return dst


def _py_mode23(cfg, chroma, interp, thr, srcs, strides, spans, shift, motions, masks, final=None):
    """render_mode23_plane_rows_inner + mode23_pixel (renderer.rs:1294-1537, :1850-1868) in plain Python."""
    cmap = lambda v: CPU_MAP[v - 1] if 1 <= v <= 32 else -1
    cd = cfg["chroma_y_div"]
    zero = not interp
    if chroma:
        W, H, BW, BH = cfg["width"] // 2, cfg["height"] // cd, cfg["block_w"] // 2, cfg["block_h"] // cd
        mox, moy = cfg["origin_x"] // 2, cfg["origin_y"] // cd
        xs_, ys_, xd, yd = cmap(cfg["block_w"] // 2), cmap(cfg["block_h"] // 2), 2, cd
    else:
        W, H, BW, BH = cfg["width"], cfg["height"], cfg["block_w"], cfg["block_h"]
        mox, moy = cfg["origin_x"], cfg["origin_y"]
        xs_, ys_, xd, yd = cmap(BW), cmap(BH), 1, 1
    ox, oy = (0, 0) if zero else (mox, moy)
    step = cfg["source_step"]
    maxx, maxy = max(W * step - 1, 0), max(H * step - 1, 0)

    def weights(total, sh):
        out = [(0, 0)] * 32
        for p in range(min(total, 32)):
            c = lambda v: int(math.ceil(v * (1 << max(sh, 0)) / total - 0.5))
            out[p] = (total - p, p) if sh < 0 else (c(total - p), c(p))
        return out

    xw, yw = weights(BW, xs_), weights(BH, ys_)
    ip = lambda a, b, total, sh, w: int((w[0] * a + w[1] * b) / total) if sh < 0 else (w[0] * a + w[1] * b) >> sh
    inv, tl = orc.render_luts(thr)
    gw, gh = cfg["grid_w"], cfg["grid_h"]
    byte = lambda v: min(max(v, 0), 255)
    b256 = lambda a, b, w: byte((a * (256 - w) + b * w) >> 8)
    b255 = lambda a, b, w: byte((a * (255 - w) + b * w + 255) >> 8)

    def index(k, x, y):
        if shift == 0:
            return y * strides[k] + x
        m = (1 << shift) - 1
        return (((y & m) << shift) | (x & m)) * spans[k] + (y >> shift) * strides[k] + (x >> shift)

    def alpha_abs(x, y, mk):
        def mat(x, y):
            i = y * gw + x
            return int(mk[i]) if x >= 0 and y >= 0 and i < len(mk) else 0
        ix0 = ix1 = iy0 = iy1 = 0
        if mox <= x:
            ix0 = (x - mox) // BW
            ix1 = ix0 + 1
        if moy <= y:
            iy0 = (y - moy) // BH
            iy1 = iy0 + 1
        fx = (x - mox) % BW if mox < x else 0
        fy = (y - moy) % BH if moy < y else 0
        top = ((BW - fx) * mat(ix0, iy0) + fx * mat(ix1, iy0)) // BW
        bot = ((BW - fx) * mat(ix0, iy1) + fx * mat(ix1, iy1)) // BW
        return byte(((BH - fy) * top + fy * bot) // BH)

    covers = all((shift == 0 or (1 << shift) == step) and index(k, maxx, maxy) < len(srcs[k]) for k in range(2))
    dst = np.zeros((H, W), dtype=np.uint8)
    for gy in range(-1, gh):
        by = 0 if gy < 0 else oy + BH * gy
        th = oy if gy < 0 else BH
        if by + BH >= H or gy == gh - 1:
            th = H - by
        th = min(by + th, H) - max(by, 0)
        if th <= 0:
            continue
        for gx in range(-1, gw):
            bx = 0 if gx < 0 else ox + BW * gx
            tw = ox if gx < 0 else BW
            if bx + BW >= W or gx == gw - 1:
                tw = W - bx
            if tw <= 0:
                continue
            i00 = max(gy, 0) * gw + max(gx, 0)
            nx = 1 if (gx >= 0 and gx != gw - 1) else 0
            ny = gw if (gy >= 0 and gy != gh - 1) else 0
            corners = [i00, i00 + nx, i00 + ny, i00 + ny + nx]
            idx = corners if interp else [i00] * 4
            S = []
            for k, (mx, my) in enumerate(motions):
                lut = inv if k & 1 else tl
                mv = lambda pl, i: int(lut[min(int(pl[i]) if i < len(pl) else 1024, 2047)])
                S.append(([int(mv(mx, i) / xd) for i in idx], [int(mv(my, i) / yd) for i in idx]))
            allx = [v for sx, _ in S for v in sx]
            ally = [v for _, sy in S for v in sy]
            direct = covers and bx * step + min(allx) >= 0 and by * step + min(ally) >= 0 and \
                (bx + tw - 1) * step + max(allx) <= maxx and (by + th - 1) * step + max(ally) <= maxy
            for y in range(th):
                wy = yw[min(y, 31)]

                def alpha_of(mk, x):
                    if zero:
                        return alpha_abs(bx + x, by + y, mk)
                    c4 = [int(mk[i]) if i < len(mk) else 0 for i in corners]
                    r = [ip(c4[0], c4[2], BH, ys_, wy), ip(c4[1], c4[3], BH, ys_, wy)]
                    return byte(ip(r[0], r[1], BW, xs_, xw[min(x, 31)]))

                for x in range(tw):
                    wx = xw[min(x, 31)]
                    vals = []
                    for k, (sx, sy) in enumerate(S):
                        if interp:
                            rx = [ip(sx[0], sx[2], BH, ys_, wy), ip(sx[1], sx[3], BH, ys_, wy)]
                            ry = [ip(sy[0], sy[2], BH, ys_, wy), ip(sy[1], sy[3], BH, ys_, wy)]
                            dx, dy = ip(rx[0], rx[1], BW, xs_, wx), ip(ry[0], ry[1], BW, xs_, wx)
                        else:
                            dx, dy = sx[0], sy[0]
                        X, Y = (bx + x) * step + dx, (by + y) * step + dy
                        if not direct:
                            X, Y = min(max(X, 0), maxx), min(max(Y, 0), maxy)
                        i = index(k & 1, X, Y)
                        vals.append(int(srcs[k & 1][i]) if i < len(srcs[k & 1]) else 0)
                    a, b, c, d = vals
                    lo, hi = min(a, b), max(a, b)
                    i0 = b255(a, min(max(d, lo), hi), alpha_of(masks[0], x))
                    i1 = b255(b, min(max(c, lo), hi), alpha_of(masks[1], x))
                    m = b256(i0, i1, thr)
                    if final is not None:
                        BX, BY = min((bx + x) * step, maxx), min((by + y) * step, maxy)
                        i, j = index(0, BX, BY), index(1, BX, BY)
                        ba = int(srcs[0][i]) if i < len(srcs[0]) else 0
                        bb = int(srcs[1][j]) if j < len(srcs[1]) else 0
                        m = b255(m, b256(ba, bb, thr), alpha_of(final, x))
                    dst[by + y, bx + x] = m
    return dst


M23_CASES = [  # w, h, block, step, interp, threshold, final mask
    (40, 24, 8, 1, True, 128, False),
    (40, 24, 16, 2, True, 60, True),
    (36, 22, 8, 1, False, 200, True),
    (20, 12, 32, 2, False, 0, False),
]


@pytest.mark.parametrize("case", range(len(M23_CASES)))
def test_oracle_mode23_matches_python_restatement(case):
    w, h, blk, step, interp, thr, with_final = M23_CASES[case]
    rng = np.random.default_rng(70 + case)
    gw, gh = _grid(w, h, blk, blk)
    cfg = _cfg(w, h, blk, blk, gw, gh, step)
    motions = [(_motion(rng, gw * gh, 40), _motion(rng, gw * gh, 40)) for _ in range(4)]
    masks = tuple(rng.integers(0, 256, size=gw * gh, dtype=np.uint8) for _ in range(2))
    final = rng.integers(0, 256, size=gw * gh, dtype=np.uint8) if with_final else None
    shift = {1: 0, 2: 1}[step]
    for chroma in (False, True):
        pw, ph = (w // 2, h // 2) if chroma else (w, h)
        strides = [pw + 1, pw + 6]
        srcs = [rng.integers(0, 256, size=(step * step) * ph * st, dtype=np.uint8) for st in strides]
        spans = [st * ph if shift else 0 for st in strides]
        got = orc.render_mode23_plane(cfg, chroma, interp, thr, srcs, strides, spans, shift, motions, masks, final,
                                      pw, ph)
        want = _py_mode23(cfg, chroma, interp, thr, srcs, strides, spans, shift, motions, masks, final)
        assert np.array_equal(got, want), f"chroma {chroma}: {np.argwhere(got != want)[:3]}"


DUAL_CASES = [  # w, h, block, step, interp, zero origin, mode, threshold, masks (0 none, 2 a+b, 3 a+b+final)
    (40, 24, 8, 1, True, False, 11, 100, 0),
    (40, 24, 8, 1, True, False, 13, 200, 2),
    (36, 22, 16, 2, False, True, 13, 64, 2),
    (32, 16, 8, 2, True, True, 11, 128, 2),    # the zero-origin variant with interpolation
    (20, 12, 32, 1, True, False, 13, 30, 0),
    (40, 24, 8, 1, True, False, 21, 150, 2),
    (40, 24, 16, 2, True, False, 22, 90, 3),
    (36, 22, 8, 1, False, True, 21, 200, 3),
    (32, 16, 8, 2, False, True, 22, 10, 2),
]


@pytest.mark.parametrize("case", range(len(DUAL_CASES)))
def test_oracle_dual_matches_python_restatement(case):
    w, h, blk, step, interp, zero, mode, thr, nmask = DUAL_CASES[case]
    rng = np.random.default_rng(50 + case)
    gw, gh = _grid(w, h, blk, blk)
    cfg = _cfg(w, h, blk, blk, gw, gh, step)
    mot0 = (_motion(rng, gw * gh, 40), _motion(rng, gw * gh, 40))
    mot1 = (_motion(rng, gw * gh, 40), _motion(rng, gw * gh, 40))
    masks = (rng.integers(0, 256, size=gw * gh, dtype=np.uint8),
             rng.integers(0, 256, size=gw * gh, dtype=np.uint8)) if nmask else None
    final = rng.integers(0, 256, size=gw * gh, dtype=np.uint8) if nmask == 3 else None
    tlimit = orc.render_threshold_limit(thr, 1.5)
    shift = {1: 0, 2: 1}[step]
    for chroma in (False, True):
        pw, ph = (w // 2, h // 2) if chroma else (w, h)
        strides = [pw + 3, pw + 5]
        srcs = [rng.integers(0, 256, size=(step * step) * ph * st, dtype=np.uint8) for st in strides]
        spans = [st * ph if shift else 0 for st in strides]
        got = orc.render_dual_plane(cfg, chroma, interp, zero, mode, thr, srcs, strides, spans, shift, mot0, mot1, pw,
                                    ph, masks, final, tlimit)
        want = _py_dual(cfg, chroma, interp, zero, mode, thr, srcs, strides, spans, shift, mot0, mot1, masks, final,
                        tlimit)
        assert np.array_equal(got, want), f"chroma {chroma}: {np.argwhere(got != want)[:3]}"


def _motion(rng, n, spread):
    m = rng.integers(1024 - spread, 1024 + spread + 1, size=n).astype(np.uint16)
    m[rng.random(n) < 0.1] = 1024
    return m


PY_CASES = [  # w, h, block, step (super clip pel), interp, threshold, mode1, mask
    (40, 24, 8, 1, True, 128, False, False),
    (40, 24, 8, 1, False, 200, True, False),
    (36, 22, 16, 1, True, 256, False, False),   # tiles stretched to the frame edge (weights past the block are 0)
    (20, 12, 32, 1, True, 90, False, False),    # blocks larger than the frame: overlapping tiles
    (32, 16, 8, 2, True, 160, True, False),     # half-pel super planes
    (24, 16, 4, 4, False, 64, False, False),    # quarter-pel super planes
    (40, 24, 8, 1, True, 128, True, True),      # masked blend (mode1_pixel), interpolated alpha
    (36, 22, 16, 2, False, 200, False, True),   # masked blend, alpha_at_absolute
]


@pytest.mark.parametrize("case", range(len(PY_CASES)))
def test_oracle_matches_python_restatement(case):
    w, h, blk, step, interp, thr, mode1, masked = PY_CASES[case]
    rng = np.random.default_rng(case)
    gw, gh = _grid(w, h, blk, blk)
    cfg = _cfg(w, h, blk, blk, gw, gh, step)
    inv, tl = orc.render_luts(thr)
    lut = inv if mode1 else tl
    mx, my = _motion(rng, gw * gh, 40), _motion(rng, gw * gh, 40)
    mask = rng.integers(0, 256, size=gw * gh, dtype=np.uint8) if masked else None
    shift = {1: 0, 2: 1, 4: 2}[step]
    for chroma in (False, True):
        pw, ph = (w // 2, h // 2) if chroma else (w, h)
        stride = pw + 3
        src = rng.integers(0, 256, size=(step * step) * ph * stride, dtype=np.uint8)
        span = stride * ph if shift else 0
        got = orc.render_warp_plane(cfg, chroma, interp, lut, src, stride, span, shift, mx, my, pw, ph, mask)
        want = _py_render(cfg, chroma, interp, lut, src, stride, span, shift, mx, my, mask)
        assert np.array_equal(got, want), f"chroma {chroma}: {np.argwhere(got != want)[:3]}"


def test_oracle_luts():
    inv, thr = orc.render_luts(77)
    s = np.arange(-1024, 1024)
    assert np.array_equal(thr, np.trunc(s * 77 / 256).astype(np.int16))
    assert np.array_equal(inv, np.trunc(s * (256 - 77) / 256).astype(np.int16))


@pytest.mark.parametrize("interp", [False, True])
def test_oracle_identity_and_shift(interp):
    w, h, blk = 64, 48, 16
    gw, gh = _grid(w, h, blk, blk)
    cfg = _cfg(w, h, blk, blk, gw, gh)
    rng = np.random.default_rng(3)
    src = rng.integers(0, 256, size=(h, w), dtype=np.uint8)
    neutral = np.full(gw * gh, 1024, np.uint16)
    _, t128 = orc.render_luts(128)
    assert np.array_equal(orc.render_warp_plane(cfg, False, interp, t128, src, w, 0, 0, neutral, neutral, w, h), src)
    _, t256 = orc.render_luts(256)  # threshold 256: the motion is the vector itself
    mx, my = np.full(gw * gh, 1024 + 5, np.uint16), np.full(gw * gh, 1024 - 3, np.uint16)
    got = orc.render_warp_plane(cfg, False, interp, t256, src, w, 0, 0, mx, my, w, h)
    ys = np.clip(np.arange(h)[:, None] - 3, 0, h - 1)
    xs = np.clip(np.arange(w)[None, :] + 5, 0, w - 1)
    assert np.array_equal(got, src[ys, xs])


@pytest.mark.parametrize("interp", [False, True])
def test_oracle_dual_known_answers(interp):
    # zero motion: both warps read the undisplaced samples a (frame 0) and b (frame 1), so
    # algorithms 11 and 13 give blend_256(a, b, t); 21 / 22 with masks 0 give blend_256(a, b, t) too
    # (blend_255(v, _, 0) = v), with masks 255 blend_256(b, a, t); 23 with its four zero sets and
    # masks 0 gives blend_256(a, b, t) again
    w, h, blk = 64, 48, 16
    gw, gh = _grid(w, h, blk, blk)
    cfg = _cfg(w, h, blk, blk, gw, gh)
    rng = np.random.default_rng(4)
    a = rng.integers(0, 256, size=(h, w), dtype=np.uint8)
    b = rng.integers(0, 256, size=(h, w), dtype=np.uint8)
    zero = (np.full(gw * gh, 1024, np.uint16), np.full(gw * gh, 1024, np.uint16))
    m0, m255 = np.zeros(gw * gh, np.uint8), np.full(gw * gh, 255, np.uint8)
    A, B = a.astype(np.int64), b.astype(np.int64)
    for t in (0, 77, 128, 256):
        want = ((A * (256 - t) + B * t) >> 8).astype(np.uint8)
        swap = ((B * (256 - t) + A * t) >> 8).astype(np.uint8)
        common = (cfg, False, interp, not interp)
        for mode in (11, 13):
            got = orc.render_dual_plane(*common, mode, t, [a, b], [w, w], [0, 0], 0, zero, zero, w, h)
            assert np.array_equal(got, want), (mode, t)
        for mode in (21, 22):
            got = orc.render_dual_plane(*common, mode, t, [a, b], [w, w], [0, 0], 0, zero, zero, w, h, (m0, m0))
            assert np.array_equal(got, want), (mode, t)
        got = orc.render_dual_plane(*common, 21, t, [a, b], [w, w], [0, 0], 0, zero, zero, w, h, (m255, m255))
        assert np.array_equal(got, swap), t
        got = orc.render_mode23_plane(cfg, False, interp, t, [a, b], [w, w], [0, 0], 0, [zero] * 4, (m0, m0), None,
                                      w, h)
        assert np.array_equal(got, want), t


def test_oracle_super_subplanes():
    # on a pel-2 super clip, a half-pel horizontal motion reads the h sub-plane at full-pel positions
    w, h, blk = 64, 48, 16
    so = orc.super_opts(w, h, "{pel:2}")
    from svpflow_b200.synth import make_clip

    frame = make_clip(w, h, 1, seed=5)[0]
    sup = orc.build_super(so, frame)
    gw, gh = _grid(w, h, blk, blk)
    cfg = _cfg(w, h, blk, blk, gw, gh, step=2)
    _, t256 = orc.render_luts(256)
    mx, my = np.full(gw * gh, 1025, np.uint16), np.full(gw * gh, 1024, np.uint16)
    luma = sup[: w * orc.super_height(so)]
    got = orc.render_warp_plane(cfg, False, True, t256, luma, w, w * h, 1, mx, my, w, h)
    hplane = luma[w * h: 2 * w * h].reshape(h, w)
    assert np.array_equal(got, hplane)


# ---------------------------------------------------------------- GPU
GPU_CASES = [  # w, h, block, step, interp, threshold, mode1, source stride pad, mask
    (1920, 1080, 16, 1, True, 128, False, 0, False),
    (1920, 1080, 16, 2, True, 96, True, 0, False),
    (1920, 1080, 8, 1, False, 256, False, 64, False),
    (640, 360, 32, 1, True, 200, True, 32, False),
    (100, 60, 8, 4, True, 40, False, 12, False),
    (66, 38, 16, 2, False, 0, True, 2, False),
    (20, 12, 32, 1, True, 175, False, 0, False),
    (1280, 720, 4, 1, True, 255, True, 0, False),
    (1920, 1080, 16, 2, True, 128, True, 0, True),
    (640, 360, 8, 1, False, 77, False, 8, True),
    (20, 12, 32, 2, True, 200, False, 0, True),
]


def _gpu_render_case(case, rng):
    import torch

    import svpflow_b200 as sv

    w, h, blk, step, interp, thr, mode1, pad, masked = case
    gw, gh = _grid(w, h, blk, blk)
    cfg = _cfg(w, h, blk, blk, gw, gh, step)
    shift = {1: 0, 2: 1, 4: 2}[step]
    mx, my = _motion(rng, gw * gh, 120), _motion(rng, gw * gh, 120)
    mask = rng.integers(0, 256, size=gw * gh, dtype=np.uint8) if masked else None
    inv, tl = orc.render_luts(thr)
    lut = inv if mode1 else tl
    srcs, wants, dsts = [], [], []
    for pl in range(3):
        pw, ph = (w // 2, h // 2) if pl else (w, h)
        stride = pw + pad
        src = rng.integers(0, 256, size=(step * step) * ph * stride, dtype=np.uint8)
        span = stride * ph if shift else 0
        wants.append(orc.render_warp_plane(cfg, pl > 0, interp, lut, src, stride, span, shift, mx, my, pw + 1, ph,
                                           mask))
        srcs.append((torch.from_numpy(src).cuda(), stride))
        dsts.append((torch.full((ph, pw + 1), 7, dtype=torch.uint8, device="cuda"), pw + 1))
    mxd = torch.from_numpy(mx.astype(np.int16)).cuda()
    myd = torch.from_numpy(my.astype(np.int16)).cuda()
    mkd = torch.from_numpy(mask).cuda() if masked else None
    sv.render_warp_device(cfg, thr, mode1, interp, [s.data_ptr() for s, _ in srcs], [st for _, st in srcs],
                          [s.numel() for s, _ in srcs], shift, mxd.data_ptr(), myd.data_ptr(),
                          [d.data_ptr() for d, _ in dsts], [st for _, st in dsts],
                          mask_ptr=mkd.data_ptr() if masked else 0)
    torch.cuda.synchronize()
    for pl in range(3):
        got = dsts[pl][0].cpu().numpy()
        want = wants[pl].copy()
        want[:, -1] = 7  # the column past the plane's width is not written
        assert np.array_equal(got, want), f"plane {pl}: {np.argwhere(got != want)[:3]}"


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(len(GPU_CASES)))
def test_render_matches_oracle(case):
    _gpu_render_case(GPU_CASES[case], np.random.default_rng(100 + case))


DUAL_GPU_CASES = [  # w, h, block, step, interp, zero origin, mode13, threshold, mask
    (1920, 1080, 16, 2, True, False, True, 128, False),
    (1920, 1080, 16, 1, True, False, False, 40, True),
    (640, 360, 8, 1, False, True, True, 200, True),
    (320, 240, 32, 2, True, True, False, 256, True),
    (66, 38, 16, 4, True, False, True, 0, False),
    (20, 12, 32, 1, True, False, True, 99, True),
]


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(len(DUAL_GPU_CASES)))
def test_render_blend_matches_oracle(case):
    import torch

    import svpflow_b200 as sv

    w, h, blk, step, interp, zero, mode13, thr, masked = DUAL_GPU_CASES[case]
    rng = np.random.default_rng(200 + case)
    gw, gh = _grid(w, h, blk, blk)
    cfg = _cfg(w, h, blk, blk, gw, gh, step)
    shift = {1: 0, 2: 1, 4: 2}[step]
    mot = [(_motion(rng, gw * gh, 150), _motion(rng, gw * gh, 150)) for _ in range(2)]
    ma = rng.integers(0, 256, size=gw * gh, dtype=np.uint8)
    mb = rng.integers(0, 256, size=gw * gh, dtype=np.uint8)
    srcs = [[], []]
    wants, dsts = [], []
    for pl in range(3):
        pw, ph = (w // 2, h // 2) if pl else (w, h)
        strides = [pw + 7 * pl, pw + 3]
        planes = [rng.integers(0, 256, size=(step * step) * ph * st, dtype=np.uint8) for st in strides]
        spans = [st * ph if shift else 0 for st in strides]
        wants.append(orc.render_dual_plane(cfg, pl > 0, interp, zero or not interp, 13 if mode13 else 11, thr, planes,
                                           strides, spans, shift, mot[0], mot[1], pw, ph, (ma, mb) if masked else None))
        for k in range(2):
            srcs[k].append((torch.from_numpy(planes[k]).cuda(), strides[k]))
        dsts.append(torch.full((ph, pw), 7, dtype=torch.uint8, device="cuda"))
    dev = lambda a: torch.from_numpy(a.astype(np.int16) if a.dtype == np.uint16 else a).cuda()
    md = [(dev(x), dev(y)) for x, y in mot]
    mkd = (dev(ma), dev(mb)) if masked else None
    sv.render_blend_device(cfg, thr, mode13, interp, zero, [t.data_ptr() for t, _ in srcs[0]],
                           [st for _, st in srcs[0]], [t.numel() for t, _ in srcs[0]],
                           [t.data_ptr() for t, _ in srcs[1]], [st for _, st in srcs[1]],
                           [t.numel() for t, _ in srcs[1]], shift, (md[0][0].data_ptr(), md[0][1].data_ptr()),
                           (md[1][0].data_ptr(), md[1][1].data_ptr()), [d.data_ptr() for d in dsts],
                           [d.shape[1] for d in dsts], masks=(mkd[0].data_ptr(), mkd[1].data_ptr()) if masked else None)
    torch.cuda.synchronize()
    for pl in range(3):
        got = dsts[pl].cpu().numpy()
        assert np.array_equal(got, wants[pl]), f"plane {pl}: {np.argwhere(got != wants[pl])[:3]}"


MASKED_GPU_CASES = [  # w, h, block, step, interp, mode22, threshold, final mask, mask scale
    (1920, 1080, 16, 2, True, False, 128, True, 1.0),
    (1920, 1080, 8, 1, True, True, 200, False, 1.5),
    (640, 360, 16, 1, False, True, 40, True, 0.75),
    (66, 38, 32, 4, True, False, 256, True, 2.0),
]


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(len(MASKED_GPU_CASES)))
def test_render_masked_matches_oracle(case):
    import torch

    import svpflow_b200 as sv

    w, h, blk, step, interp, mode22, thr, with_final, scale = MASKED_GPU_CASES[case]
    rng = np.random.default_rng(300 + case)
    gw, gh = _grid(w, h, blk, blk)
    cfg = _cfg(w, h, blk, blk, gw, gh, step)
    shift = {1: 0, 2: 1, 4: 2}[step]
    mot = [(_motion(rng, gw * gh, 150), _motion(rng, gw * gh, 150)) for _ in range(2)]
    ma, mb, mf = (rng.integers(0, 256, size=gw * gh, dtype=np.uint8) for _ in range(3))
    tlimit = orc.render_threshold_limit(thr, scale)
    srcs, wants, dsts = [[], []], [], []
    for pl in range(3):
        pw, ph = (w // 2, h // 2) if pl else (w, h)
        strides = [pw + 5, pw]
        planes = [rng.integers(0, 256, size=(step * step) * ph * st, dtype=np.uint8) for st in strides]
        spans = [st * ph if shift else 0 for st in strides]
        wants.append(orc.render_dual_plane(cfg, pl > 0, interp, not interp, 22 if mode22 else 21, thr, planes,
                                           strides, spans, shift, mot[0], mot[1], pw, ph, (ma, mb),
                                           mf if with_final else None, tlimit))
        for k in range(2):
            srcs[k].append((torch.from_numpy(planes[k]).cuda(), strides[k]))
        dsts.append(torch.full((ph, pw), 7, dtype=torch.uint8, device="cuda"))
    dev = lambda a: torch.from_numpy(a.astype(np.int16) if a.dtype == np.uint16 else a).cuda()
    md = [(dev(x), dev(y)) for x, y in mot]
    mad, mbd, mfd = dev(ma), dev(mb), dev(mf)
    sv.render_masked_device(cfg, thr, scale, mode22, interp, [t.data_ptr() for t, _ in srcs[0]],
                            [st for _, st in srcs[0]], [t.numel() for t, _ in srcs[0]],
                            [t.data_ptr() for t, _ in srcs[1]], [st for _, st in srcs[1]],
                            [t.numel() for t, _ in srcs[1]], shift, (md[0][0].data_ptr(), md[0][1].data_ptr()),
                            (md[1][0].data_ptr(), md[1][1].data_ptr()), (mad.data_ptr(), mbd.data_ptr()),
                            mfd.data_ptr() if with_final else 0, [d.data_ptr() for d in dsts],
                            [d.shape[1] for d in dsts])
    torch.cuda.synchronize()
    for pl in range(3):
        got = dsts[pl].cpu().numpy()
        assert np.array_equal(got, wants[pl]), f"plane {pl}: {np.argwhere(got != wants[pl])[:3]}"


M23_GPU_CASES = [  # w, h, block, step, interp, threshold, final mask
    (1920, 1080, 16, 2, True, 128, True),
    (1280, 720, 8, 1, True, 77, False),
    (640, 360, 16, 4, False, 200, True),
    (20, 12, 32, 1, True, 256, True),
]


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(len(M23_GPU_CASES)))
def test_render_mode23_matches_oracle(case):
    import torch

    import svpflow_b200 as sv

    w, h, blk, step, interp, thr, with_final = M23_GPU_CASES[case]
    rng = np.random.default_rng(400 + case)
    gw, gh = _grid(w, h, blk, blk)
    cfg = _cfg(w, h, blk, blk, gw, gh, step)
    shift = {1: 0, 2: 1, 4: 2}[step]
    motions = [(_motion(rng, gw * gh, 150), _motion(rng, gw * gh, 150)) for _ in range(4)]
    ma, mb, mf = (rng.integers(0, 256, size=gw * gh, dtype=np.uint8) for _ in range(3))
    srcs, wants, dsts = [[], []], [], []
    for pl in range(3):
        pw, ph = (w // 2, h // 2) if pl else (w, h)
        strides = [pw + 2, pw + 9]
        planes = [rng.integers(0, 256, size=(step * step) * ph * st, dtype=np.uint8) for st in strides]
        spans = [st * ph if shift else 0 for st in strides]
        wants.append(orc.render_mode23_plane(cfg, pl > 0, interp, thr, planes, strides, spans, shift, motions, (ma, mb),
                                             mf if with_final else None, pw, ph))
        for k in range(2):
            srcs[k].append((torch.from_numpy(planes[k]).cuda(), strides[k]))
        dsts.append(torch.full((ph, pw), 7, dtype=torch.uint8, device="cuda"))
    dev = lambda a: torch.from_numpy(a.astype(np.int16) if a.dtype == np.uint16 else a).cuda()
    md = [(dev(x), dev(y)) for x, y in motions]
    mad, mbd, mfd = dev(ma), dev(mb), dev(mf)
    sv.render_mode23_device(cfg, thr, interp, [t.data_ptr() for t, _ in srcs[0]], [st for _, st in srcs[0]],
                            [t.numel() for t, _ in srcs[0]], [t.data_ptr() for t, _ in srcs[1]],
                            [st for _, st in srcs[1]], [t.numel() for t, _ in srcs[1]], shift,
                            [(x.data_ptr(), y.data_ptr()) for x, y in md], (mad.data_ptr(), mbd.data_ptr()),
                            mfd.data_ptr() if with_final else 0, [d.data_ptr() for d in dsts], [d.shape[1] for d in dsts])
    torch.cuda.synchronize()
    for pl in range(3):
        got = dsts[pl].cpu().numpy()
        assert np.array_equal(got, wants[pl]), f"plane {pl}: {np.argwhere(got != wants[pl])[:3]}"


@pytest.mark.gpu
def test_render_after_device_chain():
    """Super -> Analyse -> vector planes -> render, all on the device, against the oracle's chain."""
    import torch

    import svpflow_b200 as sv
    from svpflow_b200.synth import make_clip

    w, h, n = 320, 240, 3
    sopt, aopt = "{pel:2}", "{block:{w:16,overlap:2},main:{search:{type:3,distance:8,satd:true}}}"
    clip = make_clip(w, h, n, seed=21, motion=6, objects=2, object_motion=8)
    sb = sv.Super(w, h, sopt)
    an = sv.Analyse(sb.sdata, aopt, w, h)
    so = orc.super_opts(w, h, sopt)
    ao = orc.analyse_opts(orc.sdata(so), aopt, None, w, h)
    sup_d = torch.empty((n, sb.output_len()), dtype=torch.uint8, device="cuda")
    pay_d = torch.empty((n, an.payload_len()), dtype=torch.uint8, device="cuda")
    scr_d = torch.empty(an.scratch_bytes(n), dtype=torch.uint8, device="cuda")
    frames_d = torch.from_numpy(clip).cuda()
    st = torch.cuda.current_stream().cuda_stream
    sb.build_device(frames_d.data_ptr(), sup_d.data_ptr(), n, st)
    an.analyse_clip_device(sup_d.data_ptr(), n, 0, n, pay_d.data_ptr(), scr_d.data_ptr(), st)
    vd = an.vector_header()
    mw, mh = sv.vector_grid(vd)
    planes = torch.empty((n, 4 * mw * mh), dtype=torch.int16, device="cuda")
    status = torch.zeros(n, dtype=torch.int32, device="cuda")
    sv.vector_planes_device(vd, pay_d.data_ptr(), an.payload_len(), n, w, h, planes.data_ptr(), status.data_ptr())
    torch.cuda.synchronize()
    sup_h = orc.build_super_many(so, clip)
    pays = orc.analyse_clip(ao, so, sup_h, 0, n)
    hs = orc.super_height(so)
    cfg = _cfg(w, h, vd[2], vd[3], mw, mh, step=2, ox=vd[2] // 2, oy=vd[3] // 2)
    offs = [0, w * hs, w * hs + (w // 2) * (hs // 2)]
    lens = [w * hs, (w // 2) * (hs // 2), (w // 2) * (hs // 2)]
    strides = [w, w // 2, w // 2]
    for f in range(n):
        mp = orc.vector_planes(vd, pays[f], w, h)
        assert np.array_equal(planes[f].cpu().numpy().view(np.uint16).reshape(4, mh, mw), mp)
        for mode1, thr in ((False, 100), (True, 100)):
            which = 1 if mode1 else 0  # mode 1 warps with the second set, mode 2 with the first
            inv, tl = orc.render_luts(thr)
            lut = inv if mode1 else tl
            dsts = [torch.zeros((h // (2 if p else 1), w // (2 if p else 1)), dtype=torch.uint8, device="cuda")
                    for p in range(3)]
            base = sup_d[f].data_ptr()
            mxp = planes[f].data_ptr() + (2 * which) * mw * mh * 2
            myp = planes[f].data_ptr() + (2 * which + 1) * mw * mh * 2
            sv.render_warp_device(cfg, thr, mode1, True, [base + o for o in offs], strides, lens, 1, mxp, myp,
                                  [d.data_ptr() for d in dsts], strides)
            torch.cuda.synchronize()
            for p in range(3):
                pw, ph = strides[p], h // (2 if p else 1)
                src = sup_h[f][offs[p]: offs[p] + lens[p]]
                want = orc.render_warp_plane(cfg, p > 0, True, lut, src, pw, pw * ph, 1, mp[2 * which],
                                             mp[2 * which + 1], pw, ph)
                assert np.array_equal(dsts[p].cpu().numpy(), want), f"frame {f} mode1 {mode1} plane {p}"


@pytest.mark.gpu
def test_render_rejects_bad_arguments():
    import svpflow_b200 as sv

    cfg = _cfg(64, 48, 16, 16, 5, 4)
    args = ([1, 1, 1], [64, 32, 32], [1, 1, 1], 0, 1, 1, [1, 1, 1], [64, 32, 32])
    with pytest.raises(ValueError, match="threshold"):
        sv.render_warp_device(cfg, 257, False, True, *args)
    with pytest.raises(ValueError, match="shift"):
        sv.render_warp_device(cfg, 10, False, True, *args[:3], 1, *args[4:])
    # odd motion-plane addresses are refused before any launch (uint16 loads there would fault)
    with pytest.raises(ValueError, match="aligned"):
        sv.render_warp_device(cfg, 10, False, True, *args[:4], 3, 3, *args[6:])
