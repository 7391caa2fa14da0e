// analyse.cu -- hierarchical block search (Analyse) on sm_100a.
//
// Restates crates/svpflow1/src/analyse_search.rs:68-2811 for the GPU:
//   * one CTA per frame pair; its two halves (NT threads each) run the forward search
//     (current -> reference) and the backward search (reference -> current). They meet
//     at a CTA barrier once per level: the forward search of a level needs the
//     backward field of the level above projected onto it, and vice versa (:128-191).
//   * inside a level the blocks run in the reference's serial order (serpentine at
//     level 0, score-sorted at coarser levels, :302-419): each block takes already
//     searched neighbours as candidates, so the order is a true dependency chain.
//   * inside a block every step of the search is a batch of candidate motion vectors
//     whose positions are known before any of them is evaluated (the special
//     candidates; a UMH cross + hexagon set; an exhaustive square; a hexagon step; an
//     expanding ring). A batch is evaluated by all NT threads as (candidate, 4x4 tile)
//     tasks, then reduced to the FIRST candidate of minimal cost below the running
//     best. That equals the reference's sequential `if cost < best.cost` scan (:1122-
//     1155) whenever cost >= motion penalty, i.e. pnew >= -256; below that the leader
//     thread replays the sequential scan over the batch's precomputed costs.
//   * a candidate's cost is a pure function of (block, vector); each candidate picks one
//     of the reference's read paths (interior, clamped, edge-shifted; :1638-2351) once,
//     and tiles then read pixels accordingly. Direct paths keep the reference's
//     wrapping index arithmetic, so out-of-range origins read what it reads.
//
// Integer/indexing work: no tensor cores, no reduced precision. The two f64 formulas
// (adapt_lambda, exact_lambda) are IEEE-exact (exact_lambda is host-precomputed).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "svpf_device.h"

namespace svpf {

namespace {

constexpr int NT = 256;        // threads per search direction
constexpr int NW = NT / 32;
constexpr int MAXC = 320;      // candidate slots per evaluation chunk
constexpr int MAXLIST = 16;    // special-candidate batch slots

enum : uint8_t { LM_DIRECT = 1, LM_SATD_MASK = 2, LM_SAD_BREAK = 3, LM_EDGE = 4, LM_DC = 5 };
enum : uint8_t { CM_NONE = 0, CM_DIRECT = 1, CM_SAD_BREAK = 3, CM_EDGE = 4 };
enum : int { BK_DONE = 0, BK_EXH, BK_UMH, BK_HEX6, BK_HEX3, BK_RING };

// status bits
constexpr int ST_PANIC = 1;      // the reference indexes out of range here (it would panic)
constexpr int ST_UNSUPPORTED = 2;

struct Cand {
    int64_t l_sbase, l_rbase, c_sbase, c_rbase;  // flat bases of the direct read paths
    int32_t l_sx, l_sy, l_rx, l_ry;              // origins of the clamped / masked paths
    int32_t c_sx, c_sy, c_rx, c_ry;
    int32_t l_srow, l_rrow, c_srow, c_rrow;      // first row of the source / reference sub-plane
    int32_t c_rows;                              // chroma rows covered (n x n for square SATD)
    uint8_t lmode, cmode, lsatd, csatd;
};

struct DirSh {
    Cand cand[MAXC];
    unsigned accL[MAXC], accU[MAXC], accV[MAXC];
    int2 mv[MAXC];
    long long motion[MAXC];
    long long kcost[MAXC];
    unsigned ksad[MAXC];
    unsigned short vlist[MAXC];
    unsigned char valid[MAXC];
    // special-candidate batch
    int lx[MAXLIST], ly[MAXLIST], lpx[MAXLIST], lpy[MAXLIST];
    unsigned char lch[MAXLIST], ldc[MAXLIST];
    unsigned resL[MAXLIST], resC[MAXLIST];
    int ln;
    // generated batch
    int bkind, bn, bcx, bcy, br, bstep, bodir;
    int nvalid;
    long long redK[NW];
    int redI[NW];
    int win;
    unsigned win_sad;
    long long best_cost;  // running best of the batch (pruning + acceptance)
    // block state shared by the search steps
    int px, py, bw, bh, chroma, pred_x, pred_y, lambda;
    int bnd[4];
    int gx, gy;           // global predictor (doubled) for the next level
    int order_len;
    int abort_;
    // reductions
    long long r64[NW][3];
    int r32[NW][2];
};

struct Planes {
    const uint8_t *y, *u, *v;
};

struct Geo {  // per level
    int lw, lh, clw, clh;
    int64_t ys, cs, ylen, clen;
};

__device__ __forceinline__ void dbar(int d) { asm volatile("bar.sync %0, %1;" ::"r"(d + 1), "r"(NT) : "memory"); }
__device__ __forceinline__ int imin(int a, int b) { return a < b ? a : b; }
__device__ __forceinline__ int imax(int a, int b) { return a > b ? a : b; }
__device__ __forceinline__ int iclamp(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
__device__ __forceinline__ unsigned sat_add(unsigned a, unsigned b) { unsigned r = a + b; return r < a ? 0xFFFFFFFFu : r; }
__device__ __forceinline__ unsigned sat_mul(unsigned a, unsigned b) {
    unsigned long long r = (unsigned long long)a * b;
    return r > 0xFFFFFFFFull ? 0xFFFFFFFFu : (unsigned)r;
}
__device__ __forceinline__ int sat_i32(long long r) {
    return r > 2147483647LL ? 2147483647 : (r < -2147483648LL ? (int)0x80000000 : (int)r);
}
__device__ __forceinline__ bool is_blk(int n) { return n == 4 || n == 8 || n == 16 || n == 32; }
// reads of a slice: an index past the end (or a wrapped, i.e. negative, one) is None
__device__ __forceinline__ unsigned rd(const uint8_t *p, int64_t len, int64_t i, unsigned dflt) {
    return (i >= 0 && i < len) ? (unsigned)__ldg(p + i) : dflt;
}
__device__ __forceinline__ long long pen(int pnew, unsigned x) { return (long long)x + (((long long)pnew * (long long)x) >> 8); }
__device__ __forceinline__ long long motion_penalty(int lambda, int px_, int py_, int mx, int my) {
    long long dx = (long long)px_ - mx, dy = (long long)py_ - my;
    return ((long long)lambda * (dx * dx + dy * dy)) >> 8;
}

// hadamard4_satd, analyse_search.rs:2681-2702
__device__ __forceinline__ unsigned hadamard4(const int d[16]) {
    int t[16];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        int s0 = d[i * 4] + d[i * 4 + 1], s1 = d[i * 4] - d[i * 4 + 1];
        int s2 = d[i * 4 + 2] + d[i * 4 + 3], s3 = d[i * 4 + 2] - d[i * 4 + 3];
        t[i * 4] = s0 + s2; t[i * 4 + 1] = s1 + s3; t[i * 4 + 2] = s0 - s2; t[i * 4 + 3] = s1 - s3;
    }
    int s = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        int s0 = t[j] + t[4 + j], s1 = t[j] - t[4 + j], s2 = t[8 + j] + t[12 + j], s3 = t[8 + j] - t[12 + j];
        s += abs(s0 + s2) + abs(s1 + s3) + abs(s0 - s2) + abs(s1 - s3);
    }
    return (unsigned)(s > 0 ? s : 0);
}

// -------------------------------------------------------------------------------------------
// Candidate set-up: the reference's choice of read path for one (block, vector).
//   edge_shift_origins :1638-1676 / block_cost_edge_lc :1996-2167
//   block_cost_luma_interior :1719-1852 / satd_luma_clamp :2353-2436
//   chroma_sad_x4 :2169-2303
__device__ void cand_setup(Cand &c, const AnalyseParams &P, const LevelInfo &L, const Geo &G, int level, int px, int py,
                           int bw, int bh, int mvx, int mvy, bool chroma, int satd, int pel_in, bool dc) {
    const int pel = imax(pel_in, 1);
    const int lw = G.lw, lh = G.lh;
    const int64_t y_off = L.y_off, c_off = L.c_off;
    if (dc) {  // block_luma_dc, :1566-1617 (a sum over the rows/columns the loop reaches)
        c.lmode = LM_DC; c.lsatd = 0; c.cmode = CM_NONE; c.csatd = 0;
        c.l_sx = px; c.l_sy = py; c.l_srow = (int32_t)y_off;
        c.c_rows = 0;
        return;
    }
    // edge_shift_origins
    const int bminx = -pel * px, bminy = -pel * py;
    const int bmaxx = pel * (lw - px - bw) + 1, bmaxy = pel * (lh - py - bh) + 1;
    const int ox = mvx < bminx ? mvx - bminx : ((bmaxx > bminx && mvx >= bmaxx) ? mvx + 1 - bmaxx : 0);
    const int oy = mvy < bminy ? mvy - bminy : ((bmaxy > bminy && mvy >= bmaxy) ? mvy + 1 - bmaxy : 0);
    const bool l0sub = level == 0 && pel >= 2;
    if (ox != 0 || oy != 0) {
        const int cx = iclamp(px - ox, 0, imax(lw - bw, 0)), cy = iclamp(py - oy, 0, imax(lh - bh, 0));
        int rx0, ry0;
        if (pel == 1) { rx0 = cx + mvx; ry0 = cy + mvy; }
        else if (pel == 4) { rx0 = (4 * cx + mvx) >> 2; ry0 = (4 * cy + mvy) >> 2; }
        else { rx0 = (2 * cx + mvx) >> 1; ry0 = (2 * cy + mvy) >> 1; }
        const int sub = l0sub ? (mvy & 1) * pel + (mvx & 1) : 0;
        c.lmode = LM_EDGE;
        c.lsatd = satd && is_blk(bw) && is_blk(bh) && bw == bh;
        c.l_sx = cx; c.l_sy = cy; c.l_rx = rx0; c.l_ry = ry0;
        c.l_srow = (int32_t)y_off; c.l_rrow = (int32_t)(y_off + (int64_t)sub * lh);
        if (chroma) {
            const int cw = bw / 2, ch = bh / 2;
            const int ccx = (px >> 1) - ((px - cx) >> 1), ccy = (py >> 1) - ((py - cy) >> 1);
            c.cmode = CM_EDGE;
            c.csatd = satd && cw == ch && (cw == 4 || cw == 8 || cw == 16);
            c.c_sx = ccx; c.c_sy = ccy;
            c.c_rx = ((mvx >> 1) + 2 * ccx) >> 1; c.c_ry = ((mvy >> 1) + 2 * ccy) >> 1;
            c.c_srow = (int32_t)c_off; c.c_rrow = (int32_t)(c_off + (int64_t)sub * G.clh);
            c.c_rows = ch;
        } else {
            c.cmode = CM_NONE; c.csatd = 0; c.c_rows = 0;
        }
        return;
    }
    // ---- luma, no edge shift
    const int px2 = px - (level > 0 && px + bw >= lw), py2 = py - (level > 0 && py + bh >= lh);
    int mx = mvx, my = mvy, sub = 0;
    if (l0sub) { sub = (mvy & 1) * pel + (mvx & 1); mx = mvx >> 1; my = mvy >> 1; }
    const uint64_t cur_row0 = (uint64_t)y_off, ref_row0 = (uint64_t)(y_off + (int64_t)sub * lh);
    const uint64_t px_u = (uint64_t)(int64_t)px2, py_u = (uint64_t)(int64_t)py2;
    c.l_srow = (int32_t)cur_row0; c.l_rrow = (int32_t)ref_row0;
    c.l_sx = px2; c.l_sy = py2; c.l_rx = px2 + mx; c.l_ry = py2 + my;
    const uint64_t ys = (uint64_t)G.ys;
    if (satd && is_blk(bw) && is_blk(bh) && bw == bh) {
        const uint64_t n = (uint64_t)bw;
        const int rx0 = px2 + mx, ry0 = py2 + my;
        auto smul = [](uint64_t a, uint64_t b) -> uint64_t { return (a != 0 && b > ~0ull / a) ? ~0ull : a * b; };
        auto sadd = [](uint64_t a, uint64_t b) -> uint64_t { uint64_t r = a + b; return r < a ? ~0ull : r; };
        const uint64_t src_end = sadd(smul(cur_row0 + py_u + n - 1, ys), px_u + n);
        const uint64_t ref_end = ry0 >= 0 ? sadd(smul(ref_row0 + (uint64_t)ry0 + n - 1, ys), (uint64_t)imax(rx0, 0) + n) : ~0ull;
        const bool interior = px_u + n <= (uint64_t)lw && py_u + n <= (uint64_t)lh && rx0 >= 0 && ry0 >= 0 &&
                              (uint64_t)rx0 + n <= (uint64_t)lw && (uint64_t)ry0 + n <= (uint64_t)lh &&
                              src_end <= (uint64_t)G.ylen && ref_end <= (uint64_t)G.ylen;
        c.lsatd = 1;
        if (interior) {
            c.lmode = LM_DIRECT;
            c.l_sbase = (int64_t)((cur_row0 + py_u) * ys + px_u);
            c.l_rbase = (int64_t)((ref_row0 + (uint64_t)ry0) * ys + (uint64_t)rx0);
        } else {
            c.lmode = LM_SATD_MASK;
        }
    } else {
        const int rx0 = px2 + mx, ry0 = py2 + my;
        const bool interior = px2 >= 0 && py2 >= 0 && rx0 >= 0 && ry0 >= 0 && px2 + bw <= lw && py2 + bh <= lh &&
                              rx0 + bw <= lw && ry0 + bh <= lh;
        c.lsatd = 0;
        if (interior && is_blk(bw)) {
            c.lmode = LM_DIRECT;
            c.l_sbase = (int64_t)((cur_row0 + py_u) * ys + px_u);
            c.l_rbase = (int64_t)((ref_row0 + (uint64_t)ry0) * ys + (uint64_t)rx0);
        } else {
            c.lmode = LM_SAD_BREAK;
        }
    }
    // ---- chroma_sad_x4
    c.cmode = CM_NONE; c.csatd = 0; c.c_rows = 0;
    if (!chroma) return;
    const int cw = bw / 2, ch = bh / 2;
    if (cw < 4 || ch < 4) return;
    const uint64_t cpx = (uint64_t)(int64_t)px / 2, cpy = (uint64_t)(int64_t)py / 2;
    const int clw = G.clw, clh = G.clh;
    int csub = 0, mcx, mcy;
    if (l0sub) { csub = (mvy & 1) * pel + (mvx & 1); mcx = mvx >> 2; mcy = mvy >> 2; }
    else { mcx = mvx >> 1; mcy = mvy >> 1; }
    const uint64_t c_cur = (uint64_t)c_off, c_ref = (uint64_t)(c_off + ((level == 0 && pel > 1) ? (int64_t)csub * clh : 0));
    const uint64_t cs = (uint64_t)G.cs;
    c.c_srow = (int32_t)c_cur; c.c_rrow = (int32_t)c_ref;
    if (cw == 4 || cw == 8 || cw == 16) {
        const int rx0 = (int)(uint32_t)cpx + mcx, ry0 = (int)(uint32_t)cpy + mcy;
        if (cpx + cw <= (uint64_t)clw && cpy + ch <= (uint64_t)clh && rx0 >= 0 && ry0 >= 0 && rx0 + cw <= clw &&
            ry0 + ch <= clh) {
            const uint64_t su = (c_cur + cpy) * cs + cpx, ru = (c_ref + (uint64_t)ry0) * cs + (uint64_t)rx0;
            if (su + (uint64_t)(ch - 1) * cs + cw <= (uint64_t)G.clen && ru + (uint64_t)(ch - 1) * cs + cw <= (uint64_t)G.clen) {
                c.cmode = CM_DIRECT;
                c.csatd = satd ? 1 : 0;
                c.c_rows = satd ? cw : ch;  // satd_interior(.., cw) reads a cw x cw square
                c.c_sbase = (int64_t)su;
                c.c_rbase = (int64_t)ru;
                return;
            }
        }
    }
    c.cmode = CM_SAD_BREAK;
    c.csatd = 0;
    c.c_rows = ch;
    c.c_sx = cpx > 0x7FFFFFFFull ? 0x7FFFFFFF : (int)cpx;
    c.c_sy = cpy > 0x7FFFFFFFull ? 0x7FFFFFFF : (int)cpy;
    c.c_rx = (int)(uint32_t)cpx + mcx;
    c.c_ry = (int)(uint32_t)cpy + mcy;
}

// One 4x4 luma tile of a candidate: its SATD, or its SAD over the part inside the block,
// or (LM_DC) the sum of its source pixels.
__device__ unsigned luma_tile(const Cand &c, const Planes &S, const Planes &R, const Geo &G, int bw, int bh, int tile) {
    const int txn = (bw + 3) >> 2;
    const int ty = tile / txn, tx = tile - ty * txn;
    const int r0 = ty * 4, c0 = tx * 4;
    const int hh = imin(4, bh - r0), ww = imin(4, bw - c0);
    const int64_t ys = G.ys, ylen = G.ylen;
    const int lw = G.lw, lh = G.lh;
    int d[16];
#pragma unroll
    for (int i = 0; i < 16; i++) d[i] = 0;
    unsigned dcsum = 0;
    switch (c.lmode) {
    case LM_DIRECT:
#pragma unroll
        for (int r = 0; r < 4; r++)
#pragma unroll
            for (int q = 0; q < 4; q++)
                if (r < hh && q < ww)
                    d[r * 4 + q] = (int)rd(S.y, ylen, c.l_sbase + (int64_t)(r0 + r) * ys + c0 + q, 0) -
                                   (int)rd(R.y, ylen, c.l_rbase + (int64_t)(r0 + r) * ys + c0 + q, 0);
        break;
    case LM_SATD_MASK:
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const int sy = c.l_sy + r0 + r;
            const int ry = iclamp(c.l_ry + r0 + r, 0, lh - 1);
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int sx = c.l_sx + c0 + q;
                const int rx = iclamp(c.l_rx + c0 + q, 0, lw - 1);
                int a = (sy >= 0 && sy < lh && sx >= 0 && sx < lw) ? (int)rd(S.y, ylen, ((int64_t)c.l_srow + sy) * ys + sx, 0) : 0;
                int b = (int)rd(R.y, ylen, ((int64_t)c.l_rrow + ry) * ys + rx, 0);
                d[r * 4 + q] = a - b;
            }
        }
        break;
    case LM_SAD_BREAK:
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const int sy = c.l_sy + r0 + r;
            const int ry = iclamp(c.l_ry + r0 + r, 0, lh - 1);
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int sx = c.l_sx + c0 + q;
                if (r < hh && q < ww && c.l_sy >= 0 && sy < lh && c.l_sx >= 0 && sx < lw) {
                    const int rx = iclamp(c.l_rx + c0 + q, 0, lw - 1);
                    d[r * 4 + q] = (int)rd(S.y, ylen, ((int64_t)c.l_srow + sy) * ys + sx, 0) -
                                   (int)rd(R.y, ylen, ((int64_t)c.l_rrow + ry) * ys + rx, 0);
                }
            }
        }
        break;
    case LM_EDGE: {
        const int mh = imax(lh - 1, 0), mw = imax(lw - 1, 0);
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const int sy = iclamp(c.l_sy + r0 + r, 0, mh), ry = iclamp(c.l_ry + r0 + r, 0, mh);
#pragma unroll
            for (int q = 0; q < 4; q++) {
                if (r < hh && q < ww) {
                    const int sx = iclamp(c.l_sx + c0 + q, 0, mw), rx = iclamp(c.l_rx + c0 + q, 0, mw);
                    d[r * 4 + q] = (int)rd(S.y, ylen, ((int64_t)c.l_srow + sy) * ys + sx, 0) -
                                   (int)rd(R.y, ylen, ((int64_t)c.l_rrow + ry) * ys + rx, 0);
                }
            }
        }
        break;
    }
    case LM_DC:
#pragma unroll
        for (int r = 0; r < 4; r++)
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int sy = c.l_sy + r0 + r, sx = c.l_sx + c0 + q;
                if (r < hh && q < ww && c.l_sy >= 0 && sy < lh && c.l_sx >= 0 && sx < lw)
                    dcsum += rd(S.y, ylen, ((int64_t)c.l_srow + sy) * ys + sx, 0);
            }
        return dcsum;
    default: return 0;
    }
    if (c.lsatd) return hadamard4(d);
    unsigned s = 0;
#pragma unroll
    for (int i = 0; i < 16; i++) s += (unsigned)abs(d[i]);
    return s;
}

// One 4x4 tile of both chroma planes of a candidate.
__device__ void chroma_tile(const Cand &c, const Planes &S, const Planes &R, const Geo &G, int cw, int tile, unsigned &ou,
                            unsigned &ov) {
    ou = 0; ov = 0;
    if (c.cmode == CM_NONE) return;
    const int txn = (cw + 3) >> 2;
    const int ty = tile / txn, tx = tile - ty * txn;
    const int r0 = ty * 4, c0 = tx * 4;
    if (r0 >= c.c_rows || c0 >= cw) return;
    const int hh = imin(4, c.c_rows - r0), ww = imin(4, cw - c0);
    const int64_t cs = G.cs, clen = G.clen;
    const int clw = G.clw, clh = G.clh;
    int du[16], dv[16];
#pragma unroll
    for (int i = 0; i < 16; i++) { du[i] = 0; dv[i] = 0; }
    if (c.cmode == CM_DIRECT) {
#pragma unroll
        for (int r = 0; r < 4; r++)
#pragma unroll
            for (int q = 0; q < 4; q++)
                if (r < hh && q < ww) {
                    const int64_t so = c.c_sbase + (int64_t)(r0 + r) * cs + c0 + q, ro = c.c_rbase + (int64_t)(r0 + r) * cs + c0 + q;
                    du[r * 4 + q] = (int)rd(S.u, clen, so, 0) - (int)rd(R.u, clen, ro, 0);
                    dv[r * 4 + q] = (int)rd(S.v, clen, so, 0) - (int)rd(R.v, clen, ro, 0);
                }
    } else if (c.cmode == CM_SAD_BREAK) {
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const long long sy = (long long)c.c_sy + r0 + r;
            const int ry = iclamp(c.c_ry + r0 + r, 0, clh - 1);
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const long long sx = (long long)c.c_sx + c0 + q;
                if (r < hh && q < ww && sy < clh && sx < clw) {
                    const int rx = iclamp(c.c_rx + c0 + q, 0, clw - 1);
                    const int64_t so = ((int64_t)c.c_srow + sy) * cs + sx, ro = ((int64_t)c.c_rrow + ry) * cs + rx;
                    du[r * 4 + q] = (int)rd(S.u, clen, so, 128) - (int)rd(R.u, clen, ro, 128);
                    dv[r * 4 + q] = (int)rd(S.v, clen, so, 128) - (int)rd(R.v, clen, ro, 128);
                }
            }
        }
    } else {  // CM_EDGE
        const int mh = imax(clh - 1, 0), mw = imax(clw - 1, 0);
        const unsigned dflt = c.csatd ? 0u : 128u;
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const int sy = iclamp(c.c_sy + r0 + r, 0, mh), ry = iclamp(c.c_ry + r0 + r, 0, mh);
#pragma unroll
            for (int q = 0; q < 4; q++)
                if (r < hh && q < ww) {
                    const int sx = iclamp(c.c_sx + c0 + q, 0, mw), rx = iclamp(c.c_rx + c0 + q, 0, mw);
                    const int64_t so = ((int64_t)c.c_srow + sy) * cs + sx, ro = ((int64_t)c.c_rrow + ry) * cs + rx;
                    du[r * 4 + q] = (int)rd(S.u, clen, so, dflt) - (int)rd(R.u, clen, ro, dflt);
                    dv[r * 4 + q] = (int)rd(S.v, clen, so, dflt) - (int)rd(R.v, clen, ro, dflt);
                }
        }
    }
    if (c.csatd) {
        ou = hadamard4(du);
        ov = hadamard4(dv);
    } else {
#pragma unroll
        for (int i = 0; i < 16; i++) { ou += (unsigned)abs(du[i]); ov += (unsigned)abs(dv[i]); }
    }
}

__device__ __forceinline__ unsigned final_luma(const Cand &c, unsigned acc) { return c.lsatd ? (acc >> 1) : acc; }
__device__ __forceinline__ unsigned final_chroma(const Cand &c, unsigned u, unsigned v) {
    if (c.cmode == CM_NONE) return 0;
    if (c.csatd) return sat_mul(sat_add(u >> 1, v >> 1), 4);
    return sat_mul(u + v, 4);
}

// -------------------------------------------------------------------------------------------
// candidate generators (the reference's loop orders)
__constant__ int2 c_hex2[8] = {{-1, -2}, {-2, 0}, {-1, 2}, {1, 2}, {2, 0}, {1, -2}, {-1, -2}, {-2, 0}};  // :889-898
__constant__ int c_mod6m1[8] = {5, 0, 1, 2, 3, 4, 5, 0};
__constant__ int2 c_hex4[16] = {{-4, 2}, {-4, 1}, {-4, 0}, {-4, -1}, {-4, -2}, {4, -2}, {4, -1}, {4, 0},
                                {4, 1},  {4, 2},  {2, 3},  {0, 4},   {-2, 3},  {-2, -3}, {0, -4}, {2, -3}};  // :1075-1092

__device__ __forceinline__ int ring_m(int r, int step) { return 2 * r > step ? (2 * r - step + step - 1) / step : 0; }

__device__ int batch_size(int kind, int r, int step) {
    switch (kind) {
    case BK_EXH: return (2 * r + 1) * (2 * r + 1);
    case BK_UMH: return 4 * (r / 2 > 0 ? r / 2 : 0) + 16 * imax(r / 4, 1);
    case BK_HEX6: return 6;
    case BK_HEX3: return 3;
    case BK_RING: return 4 * ring_m(r, step) + 4;
    }
    return 0;
}

__device__ int2 batch_mv(const DirSh &s, int i) {
    const int cx = s.bcx, cy = s.bcy, r = s.br;
    switch (s.bkind) {
    case BK_EXH: {  // exact_refine_search type 4, :799-823 (raster over the square)
        const int w = 2 * r + 1;
        return make_int2(cx - r + i % w, cy - r + i / w);
    }
    case BK_UMH: {  // exact_umh, :1055-1114
        const int nd = r / 2;
        if (i < 2 * nd) { int dd = 1 + 2 * (i >> 1); return make_int2(cx + ((i & 1) ? dd : -dd), cy); }
        i -= 2 * nd;
        if (i < 2 * nd) { int dd = 1 + 2 * (i >> 1); return make_int2(cx, cy + ((i & 1) ? dd : -dd)); }
        i -= 2 * nd;
        const int scale = 1 + i / 16;
        const int2 h = c_hex4[i % 16];
        return make_int2(cx + h.x * scale, cy + h.y * scale);
    }
    case BK_HEX6: { int2 h = c_hex2[i + 1]; return make_int2(cx + h.x, cy + h.y); }
    case BK_HEX3: { int2 h = c_hex2[s.bodir + i]; return make_int2(cx + h.x, cy + h.y); }
    case BK_RING: {  // exact_expanding, :849-885
        const int step = s.bstep, m = ring_m(r, step);
        if (i < 2 * m) { int off = -r + step + (i >> 1) * step; return make_int2(cx + off, (i & 1) ? cy + r : cy - r); }
        i -= 2 * m;
        if (i < 2 * m) { int off = -r + step + (i >> 1) * step; return make_int2((i & 1) ? cx + r : cx - r, cy + off); }
        i -= 2 * m;
        const int sx = (i < 2) ? -r : r, sy = (i & 1) ? r : -r;
        return make_int2(cx + sx, cy + sy);
    }
    }
    return make_int2(0, 0);
}

struct Ctx {
    const AnalyseParams *P;
    const LevelInfo *L;
    Geo G;
    Planes S, R;
    int level, d, tid, satd, pel;
};

// Evaluates the special-candidate batch (explicit list, per-slot block position).
__device__ void eval_list(const Ctx &x, DirSh &s) {
    const int n = s.ln;
    const int bw = s.bw, bh = s.bh;
    for (int i = x.tid; i < n; i += NT) {
        Cand &c = s.cand[i];
        cand_setup(c, *x.P, *x.L, x.G, x.level, s.lpx[i], s.lpy[i], bw, bh, s.lx[i], s.ly[i], s.lch[i] != 0, x.satd, x.pel,
                   s.ldc[i] != 0);
        s.accL[i] = 0; s.accU[i] = 0; s.accV[i] = 0;
    }
    dbar(x.d);
    const int TL = x.L->tl, TC = x.L->tc, T = TL + TC;
    const int cw = bw / 2;
    for (int t = x.tid; t < n * T; t += NT) {
        const int i = t / T, tile = t - i * T;
        const Cand &c = s.cand[i];
        if (tile < TL) {
            unsigned v = luma_tile(c, x.S, x.R, x.G, bw, bh, tile);
            if (v) atomicAdd(&s.accL[i], v);
        } else if (c.cmode != CM_NONE) {
            unsigned u, w;
            chroma_tile(c, x.S, x.R, x.G, cw, tile - TL, u, w);
            if (u) atomicAdd(&s.accU[i], u);
            if (w) atomicAdd(&s.accV[i], w);
        }
    }
    dbar(x.d);
    for (int i = x.tid; i < n; i += NT) {
        const Cand &c = s.cand[i];
        if (s.ldc[i]) { s.resL[i] = s.accL[i]; s.resC[i] = 0; continue; }
        s.resL[i] = final_luma(c, s.accL[i]);
        s.resC[i] = final_chroma(c, s.accU[i], s.accV[i]);
    }
    dbar(x.d);
}

// Evaluates a generated batch against the running best (s.best_cost). On return
// s.win is the accepted candidate (-1 if none), s.win_sad / s.best_cost its sad / cost.
__device__ void eval_gen(const Ctx &x, DirSh &s) {
    const int n = s.bn;
    const int bw = s.bw, bh = s.bh;
    const int TL = x.L->tl, TC = s.chroma ? x.L->tc : 0, T = TL + TC;
    const int cw = bw / 2;
    const int pnew = x.P->pnew;
    const bool serial = pnew < -256;
    if (x.tid == 0) s.win = -1;
    for (int base = 0; base < n; base += MAXC) {
        const int cn = imin(MAXC, n - base);
        if (x.tid == 0) s.nvalid = 0;
        dbar(x.d);
        const long long bestc = s.best_cost;
        for (int i = x.tid; i < cn; i += NT) {
            const int2 mv = batch_mv(s, base + i);
            bool ok = mv.x >= s.bnd[0] && mv.y >= s.bnd[1] && mv.x < s.bnd[2] && mv.y < s.bnd[3];
            long long motion = 0;
            if (ok) {
                motion = motion_penalty(s.lambda, s.pred_x, s.pred_y, mv.x, mv.y);
                if (motion >= bestc) ok = false;
            }
            s.mv[i] = mv;
            s.motion[i] = motion;
            s.valid[i] = ok;
            if (ok) {
                cand_setup(s.cand[i], *x.P, *x.L, x.G, x.level, s.px, s.py, bw, bh, mv.x, mv.y, s.chroma != 0, x.satd, x.pel, false);
                s.accL[i] = 0; s.accU[i] = 0; s.accV[i] = 0;
                const int slot = atomicAdd(&s.nvalid, 1);
                s.vlist[slot] = (unsigned short)i;
            }
        }
        dbar(x.d);
        const int nv = s.nvalid;
        for (int t = x.tid; t < nv * T; t += NT) {
            const int j = t / T, tile = t - j * T;
            const int i = s.vlist[j];
            const Cand &c = s.cand[i];
            if (tile < TL) {
                unsigned v = luma_tile(c, x.S, x.R, x.G, bw, bh, tile);
                if (v) atomicAdd(&s.accL[i], v);
            } else if (c.cmode != CM_NONE) {
                unsigned u, w;
                chroma_tile(c, x.S, x.R, x.G, cw, tile - TL, u, w);
                if (u) atomicAdd(&s.accU[i], u);
                if (w) atomicAdd(&s.accV[i], w);
            }
        }
        dbar(x.d);
        // finalize: cost = motion + pen(luma) + pen(chroma) (:1158-1221)
        long long bk = 0x7FFFFFFFFFFFFFFFLL;
        int bi = 0x7FFFFFFF;
        for (int i = x.tid; i < cn; i += NT) {
            if (!s.valid[i]) continue;
            const Cand &c = s.cand[i];
            const unsigned L = final_luma(c, s.accL[i]);
            const unsigned C = s.chroma ? final_chroma(c, s.accU[i], s.accV[i]) : 0u;
            const long long K = s.motion[i] + pen(pnew, L) + (s.chroma ? pen(pnew, C) : 0LL);
            s.kcost[i] = K;
            s.ksad[i] = sat_add(L, C);
            if (K < bk || (K == bk && i < bi)) { bk = K; bi = i; }
        }
        if (!serial) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                long long ok_ = __shfl_xor_sync(0xFFFFFFFFu, bk, o);
                int oi = __shfl_xor_sync(0xFFFFFFFFu, bi, o);
                if (ok_ < bk || (ok_ == bk && oi < bi)) { bk = ok_; bi = oi; }
            }
            if ((x.tid & 31) == 0) { s.redK[x.tid >> 5] = bk; s.redI[x.tid >> 5] = bi; }
        }
        dbar(x.d);
        if (x.tid == 0) {
            if (!serial) {
                long long k = s.redK[0];
                int ii = s.redI[0];
                for (int w = 1; w < NW; w++)
                    if (s.redK[w] < k || (s.redK[w] == k && s.redI[w] < ii)) { k = s.redK[w]; ii = s.redI[w]; }
                if (ii != 0x7FFFFFFF && k < s.best_cost) {
                    s.best_cost = k;
                    s.win = base + ii;
                    s.win_sad = s.ksad[ii];
                }
            } else {  // exact sequential scan (penalties may be negative)
                for (int i = 0; i < cn; i++) {
                    if (!s.valid[i]) continue;
                    if (s.motion[i] >= s.best_cost) continue;
                    if (s.kcost[i] < s.best_cost) {
                        s.best_cost = s.kcost[i];
                        s.win = base + i;
                        s.win_sad = s.ksad[i];
                    }
                }
            }
        }
        dbar(x.d);
    }
}

// -------------------------------------------------------------------------------------------
// search orders (:302-419)
__device__ __forceinline__ int64_t initial_order_len(int gw, int gh) {
    const int64_t ni = (int64_t)imax(gh - 2, 0) * imax(gw - 2, 0);
    return ni + (int64_t)gw * (gh > 1 ? 2 : 1) + (int64_t)imax(gh - 2, 0) * (gw > 1 ? 2 : 1);
}
__device__ __forceinline__ int2 initial_order_at(int gw, int gh, int64_t k) {
    const int iw = imax(gw - 2, 0);
    const int64_t ni = (int64_t)imax(gh - 2, 0) * iw;
    if (k < ni) {
        const int y = (int)(k / iw) + 1, j = (int)(k % iw);
        return make_int2((y & 1) == 0 ? 1 + j : gw - 2 - j, y);
    }
    k -= ni;
    const int64_t nb = (int64_t)gw * (gh > 1 ? 2 : 1);
    if (k < nb) {
        if (gh > 1) return make_int2((int)(k >> 1), (k & 1) ? gh - 1 : 0);
        return make_int2((int)k, 0);
    }
    k -= nb;
    if (gw > 1) return make_int2((k & 1) ? gw - 1 : 0, 1 + (int)(k >> 1));
    return make_int2(0, 1 + (int)k);
}
__device__ __forceinline__ int64_t initial_order_pos(int gw, int gh, int x, int y) {
    const int iw = imax(gw - 2, 0);
    const int64_t ni = (int64_t)imax(gh - 2, 0) * iw;
    if (y >= 1 && y <= gh - 2 && x >= 1 && x <= gw - 2)
        return (int64_t)(y - 1) * iw + ((y & 1) == 0 ? x - 1 : gw - 2 - x);
    if (y == 0) return ni + (gh > 1 ? 2 * x : x);
    if (y == gh - 1) return ni + 2 * x + 1;
    const int64_t nb = (int64_t)gw * (gh > 1 ? 2 : 1);
    if (gw > 1) return ni + nb + 2 * (int64_t)(y - 1) + (x == gw - 1 ? 1 : 0);
    return ni + nb + (y - 1);
}
// level_search_order(gw, gh, level > 0), :326-336
__device__ __forceinline__ int2 level_order_at(int gw, int gh, int64_t k) {
    const int bw = gw - 1, bh = gh - 1;
    const int64_t n0 = initial_order_len(bw, bh);
    if (k < n0) return initial_order_at(bw, bh, k);
    k -= n0;
    if (k <= bw) return make_int2((int)k, bh);
    k -= bw + 1;
    return make_int2(bw, (int)k);
}
__device__ __forceinline__ uint32_t pack_xy(int x, int y) { return (uint32_t)(x & 0xFFFF) | ((uint32_t)y << 16); }
__device__ __forceinline__ int2 unpack_xy(uint32_t v) { return make_int2((int)(v & 0xFFFF), (int)(v >> 16)); }

// -------------------------------------------------------------------------------------------
struct DirScratch {
    uint2 *vec[2];       // field per level parity: x = (u16)dx | dy << 16, y = score
    uint8_t *luma[2];
    uint2 *proj[2];
    uint32_t *order, *order2;
    int *pos;
    unsigned long long *keys;
    unsigned *hist;
    uint8_t *seen;
};
__device__ __forceinline__ int2 vmv(uint2 v) { return make_int2((int)(short)(v.x & 0xFFFF), (int)(short)(v.x >> 16)); }
__device__ __forceinline__ uint2 mkvec(int dx, int dy, unsigned score) {
    return make_uint2((uint32_t)(uint16_t)(short)dx | ((uint32_t)(uint16_t)(short)dy << 16), score);
}

// adapt_lambda, :1555-1564 (f64, IEEE-exact: one add, one division, two products)
__device__ int adapt_lambda(int nlambda, int lsad, unsigned pred_score) {
    const double l = (double)imax(lsad, 1);
    const double half = pred_score == 0xFFFFFFFFu ? -1.0 : (double)(pred_score >> 1);
    const double t = __ddiv_rn(l, __dadd_rn(l, half));
    double v = __dmul_rn(__dmul_rn((double)nlambda, t), t);
    v = fmin(v, 21474836.47);
    if (v != v) return 0;
    if (v >= 2147483647.0) return 2147483647;
    if (v <= -2147483648.0) return (int)0x80000000;
    return (int)v;
}

// block_activity / plane_activity (:1486-1553): used only when search.coarse.distance < 0.
__device__ unsigned plane_activity(const uint8_t *data, int64_t len, int64_t stride, int64_t row, int64_t x, int w, int h,
                                   bool satd) {
    const unsigned area = (unsigned)(w * h);
    unsigned sum = 0;
    for (int y = 0; y < h; y++)
        for (int c = 0; c < w; c++) sum += rd(data, len, (row + y) * stride + x + c, 0);
    const unsigned mean = area ? sum / area : 0;
    if (!satd) {
        unsigned s = 0;
        for (int y = 0; y < h; y++)
            for (int c = 0; c < w; c++) {
                unsigned v = rd(data, len, (row + y) * stride + x + c, 0);
                s += v > mean ? v - mean : mean - v;
            }
        return area ? s / area : 0;
    }
    unsigned total = 0;
    for (int y = 0; y < h; y += 4)
        for (int x0 = 0; x0 < w; x0 += 4) {
            int dd[16];
            for (int r = 0; r < 4; r++)
                for (int q = 0; q < 4; q++) dd[r * 4 + q] = (int)rd(data, len, (row + y + r) * stride + x + x0 + q, 0) - (int)mean;
            total += hadamard4(dd);
        }
    return area ? (total >> 1) / area : 0;
}

__device__ int adaptive_radius(int radius, unsigned act) {
    if (act < 2) return 0;
    unsigned a = 255u * act / 150u;
    return ((radius * (int)(a < 255 ? a : 255)) >> 8) + 1;
}

// The per-direction search of one level (exact_search_level, :480-681).
__device__ void search_level(const Ctx &x, DirSh &s, DirScratch &ds, const uint2 *prevp, int *status) {
    const AnalyseParams &P = *x.P;
    const LevelInfo &L = *x.L;
    const int level = x.level, gw = L.gw, gh = L.gh;
    const int64_t ncell = (int64_t)gw * gh;
    uint2 *field = ds.vec[level & 1];
    uint8_t *lumaf = ds.luma[level & 1];
    const int64_t order_len = s.order_len;
    // leader-only state
    int bad_count = 0;
    for (int64_t k = 0; k < order_len; k++) {
        int bx = 0, by = 0, idx = 0, edge = 0, smallest = L.smallest;
        int sxi = 0, syi = 0;
        uint2 interp = make_uint2(0, 0);
        int nseeds = 0, prev_slot = -1, rs_slot = -1, zslot = 0, gslot = 0, nslot0 = 0;
        if (x.tid == 0) {
            int2 b;
            if (level == 0) b = initial_order_at(gw, gh, k);
            else b = unpack_xy(ds.order[k]);
            bx = b.x; by = b.y;
            idx = by * gw + bx;
            int px = (level > 0 && bx == gw - 1) ? L.lw - P.block_w : bx * P.step_x;
            int py = (level > 0 && by == gh - 1) ? L.lh - P.block_h : by * P.step_y;
            px += L.pxoff; py += L.pyoff;
            s.px = px; s.py = py; s.bw = L.bw; s.bh = L.bh;
            s.bnd[0] = -L.pel * px; s.bnd[1] = -L.pel * py;
            s.bnd[2] = L.pel * (L.lw - px - L.bw) + 1; s.bnd[3] = L.pel * (L.lh - py - L.bh) + 1;
            edge = level > 0 && (bx == gw - 1 || by == gh - 1);
            sxi = imin(bx, gw - 2); syi = imin(by, gh - 2);
            const int sidx = syi * gw + sxi;
            if (sidx < 0 || (int64_t)sidx >= ncell || idx < 0 || (int64_t)idx >= ncell) {
                atomicOr(status, ST_PANIC);
                s.abort_ = 1;
            } else {
                interp = edge ? field[sidx] : field[idx];
                const int2 imv = vmv(interp);
                int n = 0;
                // slot 0: the interpolated predictor at the block
                s.lx[n] = imv.x; s.ly[n] = imv.y; s.lpx[n] = px; s.lpy[n] = py; s.lch[n] = !smallest; s.ldc[n] = 0; n++;
                // edge blocks re-score the predictor at its source block (:536-549)
                if (edge && !smallest) {
                    rs_slot = n;
                    s.lx[n] = imv.x; s.ly[n] = imv.y; s.lpx[n] = sxi * P.step_x; s.lpy[n] = syi * P.step_y;
                    s.lch[n] = 1; s.ldc[n] = 0; n++;
                }
                if (prevp) {
                    const uint2 pv = prevp[idx];
                    if (pv.y != 0xFFFFFFFFu && pv.y > 0) {
                        const int2 pm = vmv(pv);
                        prev_slot = n;
                        s.lx[n] = pm.x; s.ly[n] = pm.y; s.lpx[n] = px; s.lpy[n] = py; s.lch[n] = !smallest; s.ldc[n] = 0; n++;
                    }
                }
                zslot = n;
                s.lx[n] = 0; s.ly[n] = 0; s.lpx[n] = px; s.lpy[n] = py; s.lch[n] = !smallest; s.ldc[n] = 0; n++;  // zero
                gslot = n;
                s.lx[n] = s.gx; s.ly[n] = s.gy; s.lpx[n] = px; s.lpy[n] = py; s.lch[n] = !smallest; s.ldc[n] = 0; n++;  // global
                nslot0 = n;
                for (int ny = imax(by - 1, 0); ny <= imin(by + 1, gh - 1); ny++)
                    for (int nx = imax(bx - 1, 0); nx <= imin(bx + 1, gw - 1); nx++) {
                        const int64_t p = level == 0 ? initial_order_pos(gw, gh, nx, ny) : (int64_t)ds.pos[ny * gw + nx];
                        if (p < k) {
                            if (nseeds >= 8) { atomicOr(status, ST_PANIC); s.abort_ = 1; break; }
                            const int2 nm = vmv(field[ny * gw + nx]);
                            s.lx[n] = nm.x; s.ly[n] = nm.y; s.lpx[n] = px; s.lpy[n] = py; s.lch[n] = !smallest; s.ldc[n] = 0;
                            n++; nseeds++;
                        }
                    }
                // luma DC of the block (:1566-1617)
                s.lx[n] = 0; s.ly[n] = 0; s.lpx[n] = px; s.lpy[n] = py; s.lch[n] = 0; s.ldc[n] = 1; n++;
                s.ln = n;
                s.chroma = !smallest;
            }
        }
        dbar(x.d);
        if (s.abort_) break;
        eval_list(x, s);
        // ---- leader: exact_search_block (:684-768) on the special candidates
        int stype = 0, radius = 0, lambda = 0;
        int bmx = 0, bmy = 0, pred_x = 0, pred_y = 0;
        unsigned bsad = 0;
        long long bcost = 0;
        bool refine = false;
        if (x.tid == 0) {
            const int2 imv = vmv(interp);
            pred_x = imv.x; pred_y = imv.y;
            const unsigned pred_score = rs_slot >= 0 ? sat_add(s.resL[rs_slot], s.resC[rs_slot]) : interp.y;
            const bool field_valid = pred_score != 0xFFFFFFFFu;
            auto sadof = [&](int i) { return s.lch[i] ? sat_add(s.resL[i], s.resC[i]) : s.resL[i]; };
            if (level == 0 && P.distance == 0) {
                if (field_valid) { bmx = imv.x; bmy = imv.y; bsad = sadof(0); }
                else { bmx = 0; bmy = 0; bsad = sadof(zslot); }
            } else {
                if (field_valid) { bmx = imv.x; bmy = imv.y; bsad = sadof(0); bcost = (long long)bsad; }
                else { bmx = 0; bmy = 0; bsad = 0xFFFFFFFFu; bcost = 0x7FFFFFFFFFFFFFFFLL; }
                int ppx = imv.x, ppy = imv.y;
                if (prev_slot >= 0) {
                    const unsigned sd = sadof(prev_slot);
                    const long long cst = (long long)sd + (((long long)P.prev * sd) >> 8);
                    if (cst < bcost) { bmx = s.lx[prev_slot]; bmy = s.ly[prev_slot]; bsad = sd; bcost = cst; ppx = bmx; ppy = bmy; }
                }
                {
                    const unsigned sd = sadof(gslot);
                    const long long cst = (long long)sd + (((long long)P.pglobal * sd) >> 8);
                    if (cst < bcost) { bmx = s.lx[gslot]; bmy = s.ly[gslot]; bsad = sd; bcost = cst; }
                }
                {
                    const unsigned sd = sadof(zslot);
                    const long long cst = (long long)sd + (((long long)P.pzero * sd) >> 8);
                    if (cst < bcost) { bmx = 0; bmy = 0; bsad = sd; bcost = cst; }
                }
                for (int j = 0; j < nseeds; j++) {
                    const int i = nslot0 + j;
                    const unsigned sd = sadof(i);
                    const long long cst = (long long)sd + (((long long)P.pnbour * sd) >> 8);
                    if (cst < bcost) { bmx = s.lx[i]; bmy = s.ly[i]; bsad = sd; bcost = cst; }
                }
                bcost = (long long)bsad;
                lambda = adapt_lambda(L.lambda_base, L.lsad, pred_score);
                radius = L.base_radius;
                if (level > 0 && P.coarse_distance < 0) {
                    const int ax = s.px - (level > 0 && s.px + s.bw >= L.lw), ay = s.py - (level > 0 && s.py + s.bh >= L.lh);
                    unsigned act = plane_activity(x.S.y, x.G.ylen, x.G.ys, L.y_off + ay, ax, s.bw, s.bh, x.satd) +
                                   plane_activity(x.S.u, x.G.clen, x.G.cs, L.c_off + s.py / 2, s.px / 2, s.bw / 2, s.bh / 2, x.satd) +
                                   plane_activity(x.S.v, x.G.clen, x.G.cs, L.c_off + s.py / 2, s.px / 2, s.bw / 2, s.bh / 2, x.satd);
                    radius = adaptive_radius(radius, act);
                }
                stype = (edge && level == 1) ? 0 : L.search_type;
                refine = true;
                s.pred_x = ppx; s.pred_y = ppy;  // refinement uses the (possibly re-anchored) predictor
            }
            s.lambda = lambda;
        }
        // ---- refinement + bad-SAD expansion: leader-driven state machine, batches evaluated by all
        // states: 0 start, 1 after EXH, 2 after UMH(refine), 3 after HEX6, 4 after HEX3, 5 after hex2 ring,
        //         10 bad-start, 11 after bad ring, 12 after bad UMH, 13 after final ring, 99 store
        int st = 0, ret = 0;           // ret: where hex2 returns (0 = refine done -> bad check, 1 = bad UMH -> final ring)
        int hdir = -2, hi = 1, hbx = 0, hby = 0, hrad = 0, bad_r = 0, bad_max = 0;
        unsigned found = 0;
        if (x.tid == 0) st = refine ? 0 : 10;
        for (;;) {
            if (x.tid == 0) {
                int issue = BK_DONE;
                for (;;) {  // advance until a batch is issued or the block is done
                    if (st == 0) {
                        if (stype == 4) { s.bkind = BK_EXH; s.bcx = bmx; s.bcy = bmy; s.br = radius; issue = 1; st = 1; }
                        else if (stype == 3) { s.bkind = BK_UMH; s.bcx = bmx; s.bcy = bmy; s.br = radius; issue = 1; st = 2; }
                        else if (stype == 2) { st = 20; ret = 0; hrad = radius; }
                        else st = 10;
                    } else if (st == 1) { st = 10; }
                    else if (st == 2) { st = 20; ret = 0; hrad = radius; }
                    else if (st == 20) {  // exact_hex2 entry (:942-1033)
                        hbx = bmx; hby = bmy;
                        if (hrad > 1) { hdir = -2; s.bkind = BK_HEX6; s.bcx = hbx; s.bcy = hby; issue = 1; st = 3; }
                        else { s.bkind = BK_RING; s.bcx = hbx; s.bcy = hby; s.br = 1; s.bstep = 1; issue = 1; st = 5; }
                    } else if (st == 21) {  // hex2 iteration test
                        if (hi < hrad / 2 && hbx >= s.bnd[0] && hby >= s.bnd[1] && hbx < s.bnd[2] && hby < s.bnd[3]) {
                            const int odir = c_mod6m1[hdir + 1];
                            s.bodir = odir; s.bkind = BK_HEX3; s.bcx = hbx; s.bcy = hby; issue = 1; st = 4;
                        } else st = 22;
                    } else if (st == 22) {  // hex2 exit: best.mv = (bmx, bmy), then radius-1 ring
                        bmx = hbx; bmy = hby;
                        s.bkind = BK_RING; s.bcx = hbx; s.bcy = hby; s.br = 1; s.bstep = 1; issue = 1; st = 5;
                    } else if (st == 5) { st = ret == 0 ? 10 : 13; if (ret == 1) { s.bkind = BK_RING; s.bcx = bmx; s.bcy = bmy; s.br = 1; s.bstep = 1; issue = 1; st = 13; } }
                    else if (st == 10) {  // bad-SAD expansion, :611-672
                        found = bsad;
                        const int bl = sat_i32((long long)P.coarse_bad_sad + (long long)(sat_i32((long long)P.coarse_bad_sad * bad_count) / 16));
                        if (refine && level > 0 && idx > 1 && P.coarse_bad_sad > 0 && (int)bsad > bl) {
                            bad_count++;
                            s.pred_x = pred_x; s.pred_y = pred_y;  // the block's own predictor
                            if (P.coarse_bad_range < 0) {
                                bad_max = -P.coarse_bad_range * L.pel; bad_r = L.pel;
                                if (bad_r < bad_max) { s.bkind = BK_RING; s.bcx = 0; s.bcy = 0; s.br = bad_r; s.bstep = L.pel; issue = 1; st = 11; }
                                else { s.bkind = BK_RING; s.bcx = bmx; s.bcy = bmy; s.br = 1; s.bstep = 1; issue = 1; st = 13; }
                            } else if (P.coarse_bad_range > 0) {
                                s.bkind = BK_UMH; s.bcx = 0; s.bcy = 0; s.br = P.coarse_bad_range * L.pel; hrad = s.br; issue = 1; st = 12;
                            } else {
                                s.bkind = BK_RING; s.bcx = bmx; s.bcy = bmy; s.br = 1; s.bstep = 1; issue = 1; st = 13;
                            }
                        } else st = 99;
                    } else if (st == 11) {
                        if (bsad < found / 4) st = 14;
                        else {
                            bad_r += L.pel;
                            if (bad_r < bad_max) { s.bkind = BK_RING; s.bcx = 0; s.bcy = 0; s.br = bad_r; s.bstep = L.pel; issue = 1; st = 11; }
                            else st = 14;
                        }
                    } else if (st == 14) { s.bkind = BK_RING; s.bcx = bmx; s.bcy = bmy; s.br = 1; s.bstep = 1; issue = 1; st = 13; }
                    else if (st == 12) { st = 20; ret = 1; }
                    else if (st == 13) { st = 99; }
                    else { st = 99; }
                    if (issue || st == 99) break;
                }
                if (!issue) s.bkind = BK_DONE;
                else { s.best_cost = bcost; s.bn = batch_size(s.bkind, s.br, s.bkind == BK_RING ? s.bstep : 1); }
            }
            dbar(x.d);
            if (s.bkind == BK_DONE) break;
            eval_gen(x, s);
            if (x.tid == 0) {
                const int w = s.win;
                const int kind = s.bkind;
                if (w >= 0) {
                    bsad = s.win_sad;
                    bcost = s.best_cost;
                    if (kind == BK_HEX6 || kind == BK_HEX3) {
                        hdir = kind == BK_HEX6 ? w : s.bodir + w - 1;  // check_dir label; best.mv is set at hex2 exit
                    } else {
                        const int2 mv = batch_mv(s, w);
                        bmx = mv.x; bmy = mv.y;
                    }
                }
                if (kind == BK_HEX6) {
                    if (w >= 0) {
                        hbx += c_hex2[hdir + 1].x; hby += c_hex2[hdir + 1].y; hi = 1; st = 21;
                    } else st = 22;
                } else if (kind == BK_HEX3) {
                    if (w >= 0) { hbx += c_hex2[hdir + 1].x; hby += c_hex2[hdir + 1].y; hi++; st = 21; }
                    else st = 22;
                }
            }
        }
        // ---- store (:673-679)
        if (x.tid == 0) {
            const int ln = s.ln - 1;  // the DC slot
            const int rows = (s.py >= 0) ? imax(0, imin(s.bh, L.lh - s.py)) : 0;
            const int cols = (s.px >= 0) ? imax(0, imin(s.bw, L.lw - s.px)) : 0;
            const unsigned cnt = (unsigned)(rows * cols);
            unsigned dc = cnt ? s.resL[ln] / cnt : 0;
            if (dc > 255) dc = 255;
            field[idx] = mkvec(bmx, bmy, smallest ? sat_mul(bsad, 3) : bsad);
            lumaf[idx] = (uint8_t)dc;
        }
        // the next block's leader reads field[] written above by the same thread: no barrier needed
    }
}

// exact_global_doubled (:1285-1324) over the dir's threads
__device__ void global_doubled(const Ctx &x, DirSh &s, const uint2 *field, int64_t n, unsigned *hist) {
    int mode[2];
    for (int comp = 0; comp < 2; comp++) {
        int mn = 0x7FFFFFFF, mx = (int)0x80000000;
        for (int64_t i = x.tid; i < n; i += NT) {
            const int2 v = vmv(field[i]);
            const int c = comp == 0 ? v.x : v.y;
            mn = imin(mn, c); mx = imax(mx, c);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) { mn = imin(mn, __shfl_xor_sync(~0u, mn, o)); mx = imax(mx, __shfl_xor_sync(~0u, mx, o)); }
        if ((x.tid & 31) == 0) { s.r32[x.tid >> 5][0] = mn; s.r32[x.tid >> 5][1] = mx; }
        dbar(x.d);
        mn = s.r32[0][0]; mx = s.r32[0][1];
        for (int w = 1; w < NW; w++) { mn = imin(mn, s.r32[w][0]); mx = imax(mx, s.r32[w][1]); }
        dbar(x.d);
        if (n == 0) { mode[comp] = 0; continue; }
        for (int v = mn + x.tid; v <= mx; v += NT) hist[v + 32768] = 0;
        dbar(x.d);
        for (int64_t i = x.tid; i < n; i += NT) {
            const int2 v = vmv(field[i]);
            atomicAdd(&hist[(comp == 0 ? v.x : v.y) + 32768], 1u);
        }
        dbar(x.d);
        // most frequent value, the smallest one among ties
        unsigned bc = 0;
        int bv = 0x7FFFFFFF;
        for (int v = mn + x.tid; v <= mx; v += NT) {
            const unsigned c = hist[v + 32768];
            if (c > bc || (c == bc && v < bv)) { bc = c; bv = v; }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            unsigned oc = __shfl_xor_sync(~0u, bc, o);
            int ov = __shfl_xor_sync(~0u, bv, o);
            if (oc > bc || (oc == bc && ov < bv)) { bc = oc; bv = ov; }
        }
        if ((x.tid & 31) == 0) { s.r32[x.tid >> 5][0] = (int)bc; s.r32[x.tid >> 5][1] = bv; }
        dbar(x.d);
        bc = (unsigned)s.r32[0][0]; bv = s.r32[0][1];
        for (int w = 1; w < NW; w++) {
            const unsigned oc = (unsigned)s.r32[w][0];
            const int ov = s.r32[w][1];
            if (oc > bc || (oc == bc && ov < bv)) { bc = oc; bv = ov; }
        }
        mode[comp] = bv;
        dbar(x.d);
    }
    long long sx = 0, sy = 0, cnt = 0;
    for (int64_t i = x.tid; i < n; i += NT) {
        const int2 v = vmv(field[i]);
        if (abs(v.x - mode[0]) < 6 && abs(v.y - mode[1]) < 6) { sx += v.x; sy += v.y; cnt++; }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sx += __shfl_xor_sync(~0u, sx, o); sy += __shfl_xor_sync(~0u, sy, o); cnt += __shfl_xor_sync(~0u, cnt, o);
    }
    if ((x.tid & 31) == 0) { s.r64[x.tid >> 5][0] = sx; s.r64[x.tid >> 5][1] = sy; s.r64[x.tid >> 5][2] = cnt; }
    dbar(x.d);
    if (x.tid == 0) {
        sx = 0; sy = 0; cnt = 0;
        for (int w = 0; w < NW; w++) { sx += s.r64[w][0]; sy += s.r64[w][1]; cnt += s.r64[w][2]; }
        if (cnt == 0) { s.gx = 2 * mode[0]; s.gy = 2 * mode[1]; }
        else {
            const long long ssx = (sx > 0) - (sx < 0), ssy = (sy > 0) - (sy < 0);
            s.gx = 2 * (int)((sx + ssx * cnt / 2) / cnt);
            s.gy = 2 * (int)((sy + ssy * cnt / 2) / cnt);
        }
    }
    dbar(x.d);
}

// reorder_search_order (:404-419): stable sort of the interior cells by score >> shift
__device__ void reorder(const Ctx &x, DirSh &s, const uint2 *field, int gw, int gh, DirScratch &ds, int *status) {
    const int64_t count = (int64_t)(gw - 1) * (gh - 1);
    if (count > s.order_len) {
        if (x.tid == 0) { atomicOr(status, ST_PANIC); s.abort_ = 1; }
        dbar(x.d);
        return;
    }
    unsigned v = (unsigned)imax(x.P->block_w * x.P->block_h / 8, 1), lg = 0;
    while (v >>= 1) lg++;
    const unsigned shift = lg + 1;
    int64_t np = 1;
    while (np < count) np <<= 1;
    unsigned long long *keys = ds.keys;
    for (int64_t i = x.tid; i < np; i += NT) {
        if (i < count) {
            const int xx = (int)(i % (gw - 1)), yy = (int)(i / (gw - 1));
            keys[i] = ((unsigned long long)(field[(int64_t)yy * gw + xx].y >> shift) << 32) | (unsigned long long)i;
        } else {
            keys[i] = ~0ull;
        }
    }
    dbar(x.d);
    for (int64_t kk = 2; kk <= np; kk <<= 1)
        for (int64_t j = kk >> 1; j > 0; j >>= 1) {
            for (int64_t i = x.tid; i < np; i += NT) {
                const int64_t l = i ^ j;
                if (l > i) {
                    const unsigned long long a = keys[i], b = keys[l];
                    const bool up = (i & kk) == 0;
                    if ((a > b) == up) { keys[i] = b; keys[l] = a; }
                }
            }
            dbar(x.d);
        }
    for (int64_t i = x.tid; i < count; i += NT) {
        const unsigned r = (unsigned)(keys[i] & 0xFFFFFFFFull);
        ds.order[i] = pack_xy((int)(r % (unsigned)(gw - 1)), (int)(r / (unsigned)(gw - 1)));
    }
    dbar(x.d);
}

__global__ void __launch_bounds__(2 * NT, 1)
    analyse_kernel(const __grid_constant__ AnalyseParams P, const PairSrc psrc, uint8_t *__restrict__ payloads,
                   uint8_t *__restrict__ scratch, int *status) {
    extern __shared__ __align__(16) unsigned char smem[];
    const bool bidir = P.vectors == 3;
    const int half = bidir ? (int)(threadIdx.x / NT) : 0;
    const int d = bidir ? half : ((P.vectors & 2) ? 0 : 1);  // 0 = forward (cur -> ref), 1 = backward
    const int tid = threadIdx.x % NT;
    DirSh &s = reinterpret_cast<DirSh *>(smem)[half];
    __shared__ int cta_abort;
    const int64_t pair = blockIdx.x;
    PairRef pr;
    if (psrc.table) {
        pr = psrc.table[pair];
    } else {  // analyse_filter.rs:277-282: frame n pairs with min(n + delta, num_frames - 1)
        const int64_t n = (int64_t)psrc.first + pair;
        int64_t n2 = n + psrc.delta;
        if (n2 > psrc.nframes - 1) n2 = psrc.nframes - 1;
        pr.cur = psrc.clip + n * psrc.frame_bytes;
        pr.ref = psrc.clip + n2 * psrc.frame_bytes;
    }
    const uint8_t *src = d == 0 ? pr.cur : pr.ref;
    const uint8_t *ref = d == 0 ? pr.ref : pr.cur;
    uint8_t *scr = scratch + pair * P.scratch_per_pair;
    DirScratch ds;
    ds.vec[0] = (uint2 *)(scr + P.off_field[d]);
    ds.vec[1] = (uint2 *)(scr + P.off_next[d]);
    ds.luma[0] = scr + P.off_out[d];
    ds.luma[1] = scr + P.off_out[d] + P.max_cells;
    ds.proj[0] = (uint2 *)(scr + P.off_proj[d][0]);
    ds.proj[1] = (uint2 *)(scr + P.off_proj[d][1]);
    ds.order = (uint32_t *)(scr + P.off_order[d]);
    ds.order2 = (uint32_t *)(scr + P.off_order2[d]);
    ds.pos = (int *)(scr + P.off_pos[d]);
    ds.keys = (unsigned long long *)(scr + P.off_keys[d]);
    ds.hist = (unsigned *)(scr + P.off_hist[d]);
    ds.seen = scr + P.off_seen[d];
    Ctx x;
    x.P = &P;
    x.d = half;
    x.tid = tid;
    x.S = Planes{src, src + P.y_len, src + P.y_len + P.c_len};
    x.R = Planes{ref, ref + P.y_len, ref + P.y_len + P.c_len};
    if (threadIdx.x == 0) cta_abort = 0;
    if (tid == 0) { s.abort_ = 0; s.gx = 0; s.gy = 0; s.order_len = 0; }
    __syncthreads();
    const uint2 *other_proj[2] = {nullptr, nullptr};
    {
        const int od = bidir ? 1 - d : d;
        other_proj[0] = (const uint2 *)(scr + P.off_proj[od][0]);
        other_proj[1] = (const uint2 *)(scr + P.off_proj[od][1]);
    }
    int pgw = 0, pgh = 0;  // grid of the previous (coarser) level
    for (int level = P.nlevels - 1; level >= 0; level--) {
        const LevelInfo &L = P.lv[level];
        x.L = &L;
        x.level = level;
        x.satd = L.satd;
        x.pel = L.pel;
        x.G.lw = L.lw; x.G.lh = L.lh; x.G.clw = L.lw / 2; x.G.clh = L.lh / 2;
        x.G.ys = P.y_stride; x.G.cs = P.c_stride; x.G.ylen = P.y_len; x.G.clen = P.c_len;
        const int gw = L.gw, gh = L.gh;
        const int64_t ncell = (int64_t)gw * gh;
        const bool first = level == P.nlevels - 1;
        if (!s.abort_) {
            // ---- search order of this level
            if (level == 0) {
                if (tid == 0) s.order_len = (int)initial_order_len(gw, gh);
            } else if (first) {
                const int64_t n0 = initial_order_len(gw - 1, gh - 1) + gw + (gh - 1);
                for (int64_t k = tid; k < n0; k += NT) {
                    const int2 b = level_order_at(gw, gh, k);
                    ds.order[k] = pack_xy(b.x, b.y);
                }
                if (tid == 0) s.order_len = (int)n0;
            } else {  // refine_search_order (:338-402), serial
                for (int64_t i = tid; i < ncell; i += NT) ds.seen[i] = 0;
                dbar(half);
                if (tid == 0) {
                    const int sw = pgw - 1, sh = pgh - 1, dw = gw - 1, dh = gh - 1;
                    const int ex = imax(dw - 2 * sw, 0), ey = imax(dh - 2 * sh, 0);
                    int64_t ni = 0, nb = 0;
                    uint32_t *bnd = (uint32_t *)ds.keys;  // boundary list
                    auto add = [&](int cx, int cy) {
                        if (cx < 0 || cy < 0 || cx >= dw || cy >= dh) return;
                        const int64_t ix = (int64_t)cy * gw + cx;
                        if (ds.seen[ix]) return;
                        ds.seen[ix] = 1;
                        if (cx > 0 && cy > 0 && cx < dw - 1 && cy < dh - 1) ds.order2[ni++] = pack_xy(cx, cy);
                        else bnd[nb++] = pack_xy(cx, cy);
                    };
                    for (int64_t k = 0; k < s.order_len; k++) {
                        const int2 c = unpack_xy(ds.order[k]);
                        if (c.x >= sw || c.y >= sh) continue;
                        const int left = 2 * c.x, top = 2 * c.y;
                        add(left, top); add(left + 1, top); add(left + 1, top + 1); add(left, top + 1);
                        if (c.x == sw - 1)
                            for (int dx = 2; dx < 2 + ex; dx++)
                                for (int dy = 0; dy < 2 + (c.y == sh - 1) * ey; dy++) add(left + dx, top + dy);
                        if (c.y == sh - 1)
                            for (int dy = 2; dy < 2 + ey; dy++)
                                for (int dx = 0; dx < 2; dx++) add(left + dx, top + dy);
                    }
                    for (int64_t i = 0; i < nb; i++) ds.order2[ni++] = bnd[i];
                    for (int xx = 0; xx <= dw; xx++) ds.order2[ni++] = pack_xy(xx, dh);
                    for (int yy = 0; yy < dh; yy++) ds.order2[ni++] = pack_xy(dw, yy);
                    s.order_len = (int)ni;
                }
                dbar(half);
                for (int64_t k = tid; k < s.order_len; k += NT) ds.order[k] = ds.order2[k];
            }
            dbar(half);
            if (level > 0) {  // first position of every cell in the order ("processed" test)
                for (int64_t i = tid; i < ncell; i += NT) ds.pos[i] = 0x7FFFFFFF;
                dbar(half);
                for (int64_t k = tid; k < s.order_len; k += NT) {
                    const int2 c = unpack_xy(ds.order[k]);
                    atomicMin(&ds.pos[(int64_t)c.y * gw + c.x], (int)k);
                }
            }
            // ---- interpolate the coarser field (:421-478), or start from zeros
            uint2 *nf = ds.vec[level & 1];
            uint8_t *nl = ds.luma[level & 1];
            uint2 *pj = ds.proj[level & 1];
            if (first) {
                for (int64_t i = tid; i < ncell; i += NT) { nf[i] = make_uint2(0, 0); nl[i] = 0; }
            } else {
                const uint2 *cf = ds.vec[(level + 1) & 1];
                const uint8_t *cl = ds.luma[(level + 1) & 1];
                const int cw = pgw - 1, ch = pgh - 1, pel = L.pel;
                for (int64_t i = tid; i < ncell; i += NT) {
                    const int xx = (int)(i % gw), yy = (int)(i / gw);
                    uint2 out = make_uint2(0, 0);
                    uint8_t ol = 0;
                    if (xx < gw - 1 && yy < gh - 1) {
                        int64_t ci;
                        if (xx < 2 * cw && yy < 2 * ch) ci = (int64_t)(yy >> 1) * pgw + (xx >> 1);
                        else {
                            const int e = ch + imin(xx >> 1, cw) - imin(yy >> 1, ch);
                            ci = e <= cw ? (int64_t)ch * pgw + e : (int64_t)(cw + ch - e) * pgw + cw;
                        }
                        const uint2 p = cf[ci];
                        const int2 pm = vmv(p);
                        out = mkvec(iclamp(pm.x * 2 * pel, -32768, 32767), iclamp(pm.y * 2 * pel, -32768, 32767), p.y);
                        ol = cl[ci];
                    }
                    nf[i] = out;
                    nl[i] = ol;
                    ds.keys[i] = ~0ull;
                }
                dbar(half);
                for (int64_t i = tid; i < ncell; i += NT) {
                    const int xx = (int)(i % gw), yy = (int)(i / gw);
                    if (xx >= gw - 1 || yy >= gh - 1 || xx >= 2 * cw || yy >= 2 * ch) continue;
                    const uint2 p = cf[(int64_t)(yy >> 1) * pgw + (xx >> 1)];
                    if (p.y == 0xFFFFFFFFu) continue;  // `score < target.score` never holds
                    const int2 pm = vmv(p);
                    const int vx = pm.x * 2 * pel, vy = pm.y * 2 * pel;
                    const int bw = P.block_w, bh = P.block_h;
                    const int tx = iclamp((vx + (bw >> 1) + (bw - P.ox) * xx) / (bw - P.ox), 0, gw - 1);
                    const int ty = iclamp((vy + (bh >> 1) + (bh - P.oy) * yy) / (bh - P.oy), 0, gh - 1);
                    atomicMin(&ds.keys[(int64_t)ty * gw + tx], ((unsigned long long)p.y << 32) | (unsigned long long)i);
                }
                dbar(half);
                for (int64_t i = tid; i < ncell; i += NT) {
                    const unsigned long long kk = ds.keys[i];
                    if (kk == ~0ull) pj[i] = make_uint2(0, 0xFFFFFFFFu);
                    else {
                        const uint2 v = nf[kk & 0xFFFFFFFFull];
                        const int2 m = vmv(v);
                        pj[i] = mkvec(-m.x, -m.y, v.y);
                    }
                }
            }
        }
        __syncthreads();  // both directions' projections of this level are ready
        if (!s.abort_) {
            const uint2 *prevp = (first) ? nullptr : other_proj[level & 1];
            search_level(x, s, ds, prevp, status);
        }
        dbar(half);
        if (!s.abort_ && level > 0) {
            const uint2 *f = ds.vec[level & 1];
            global_doubled(x, s, f, ncell, ds.hist);
            reorder(x, s, f, gw, gh, ds, status);
        }
        pgw = gw; pgh = gh;
        if (tid == 0 && s.abort_) cta_abort = 1;
        __syncthreads();
    }
    if (cta_abort) return;
    // ---- refine pass (exact_recalculate :1326-1451) runs on the host-selected configs only
    // ---- rescale_scores (:2716-2738) + pack_vector_frame (:2740-2811)
    const uint2 *f = ds.vec[0];
    const uint8_t *fl = ds.luma[0];
    const int64_t count = (int64_t)P.out_gw * P.out_gh;
    uint8_t *pay = payloads + pair * P.payload_len;
    const int64_t region = bidir ? (d == 1 ? 0x40 : 0x40 + 4 + count * 8) : 0x40;
    if (threadIdx.x == 0) {
        for (int i = 0; i < 16; i++) reinterpret_cast<int *>(pay)[i] = P.header[i];
    }
    if (tid == 0) *reinterpret_cast<int *>(pay + region) = (int)(2 * count + 1);
    for (int64_t i = tid; i < count; i += NT) {
        const uint2 v = f[i];
        const int2 m = vmv(v);
        const int mag = abs(m.x) + abs(m.y);
        const int ratio = (100 * mag) / P.rescale_denom;
        int score = (int)v.y;
        if (ratio >= 51) score = sat_i32((long long)score * 20);
        else if (ratio >= 16) {
            const unsigned long long v71 = (3926827243ull * (unsigned long long)(unsigned)score * (unsigned long long)(unsigned)(ratio - 15)) >> 32;
            const int w = (int)(unsigned)v71;
            score = sat_i32((long long)score + 9 * ((w >> 31) + (w >> 5)));
        }
        const unsigned sc = (unsigned)score & 0x00FFFFFFu;
        uint8_t *o = pay + region + 4 + i * 8;
        const unsigned d0 = ((unsigned)(int)m.x << 16) | (unsigned)(uint16_t)(short)m.y;
        const unsigned d1 = sc | ((unsigned)fl[i] << 24);
        memcpy(o, &d0, 4);
        memcpy(o + 4, &d1, 4);
    }
}

}  // namespace

cudaError_t launch_analyse(const AnalyseParams &P, const PairSrc &psrc, int npairs, uint8_t *payloads,
                           uint8_t *scratch, int *status_dev, cudaStream_t stream, int *launches) {
    if (npairs <= 0) return cudaSuccess;
    const int ndir = P.vectors == 3 ? 2 : 1;
    const size_t smem = sizeof(DirSh) * ndir;
    static bool attr_set = false;
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(analyse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(2 * sizeof(DirSh)));
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    analyse_kernel<<<npairs, NT * ndir, smem, stream>>>(P, psrc, payloads, scratch, status_dev);
    if (launches) *launches += 1;
    return cudaGetLastError();
}

size_t analyse_dir_shared_bytes() { return sizeof(DirSh); }

// -------------------------------------------------------------------------------------------
bool build_analyse_params(const AnalyseOpts &o, const SuperLayout &Lay, AnalyseParams &P, std::string &err) {
    memset(&P, 0, sizeof(P));
    if (o.levels < 1 || o.levels > kMaxLevels) { err = "unsupported level count"; return false; }
    if (!Lay.full) { err = "SVAnalyse: the super clip must hold the finest level (full=true)"; return false; }
    P.nlevels = o.levels;
    P.block_w = o.block_w; P.block_h = o.block_h; P.ox = o.overlap_x; P.oy = o.overlap_y;
    P.step_x = o.block_w - o.overlap_x > 1 ? o.block_w - o.overlap_x : 1;
    P.step_y = o.block_h - o.overlap_y > 1 ? o.block_h - o.overlap_y : 1;
    P.pnew = o.pnew; P.prev = o.prev; P.pzero = o.pzero; P.pglobal = o.pglobal; P.pnbour = o.pnbour;
    P.distance = o.distance; P.coarse_bad_sad = o.coarse_bad_sad; P.coarse_bad_range = o.coarse_bad_range;
    P.coarse_distance = o.coarse_distance; P.vectors = o.vectors;
    P.luma_w = o.width; P.luma_h = o.height; P.pel = o.pel;
    P.y_stride = Lay.y_stride; P.c_stride = Lay.c_stride; P.y_len = Lay.y_len; P.c_len = Lay.c_len;
    P.frame_bytes = Lay.frame_bytes;
    P.lambda = o.lambda;
    // per level
    int64_t max_cells = 1, max_order = 1;
    for (int lv = 0; lv < o.levels; lv++) {
        LevelInfo &L = P.lv[lv];
        level_grid(o, lv, L.gw, L.gh);
        L.lw = reduce_dim(o.width, lv);
        L.lh = reduce_dim(o.height, lv);
        int64_t y = 0, c = 0;  // level_y_offset / chroma_level_offset (:49-58, :2704-2713)
        for (int k = 0; k < lv; k++) {
            const int64_t h = reduce_dim(Lay.height, k);
            const int64_t sub = (k == 0 && Lay.full) ? (int64_t)Lay.pel * Lay.pel : 1;
            y += h * sub;
            const int64_t hc = h / 2;
            c += (hc > 1 ? hc : 1) * sub;
        }
        L.y_off = y; L.c_off = c;
        L.pel = lv == 0 ? (o.pel > 1 ? o.pel : 1) : 1;
        L.smallest = lv == o.levels - 1;
        // exact_lambda (:1279-1283), f64: lambda / plevel^(levels-level-1) / pel^2
        {
            double a = o.plevel, r = 1.0;
            int b = o.levels - lv - 1;
            for (;;) {  // compiler-rt __powidf2 order
                if (b & 1) r *= a;
                b /= 2;
                if (b == 0) break;
                a *= a;
            }
            const double v = (double)o.lambda / r / (double)((L.pel * L.pel) > 1 ? L.pel * L.pel : 1);
            int32_t iv;
            if (v != v) iv = 0;
            else if (v >= 2147483647.0) iv = INT32_MAX;
            else if (v <= -2147483648.0) iv = INT32_MIN;
            else iv = (int32_t)v;
            L.lambda_base = L.smallest ? 0 : iv;
        }
        L.lsad = L.smallest ? o.lsad / 3 : o.lsad;
        L.satd = lv == 0 ? o.fine_satd : o.coarse_satd;
        L.search_type = lv == 0 ? o.search_type : o.coarse_search_type;
        {  // search_radius (:1465-1476)
            const int dd = lv == 0 ? o.distance : o.coarse_distance;
            const int nl = o.levels > 1 ? o.levels : 1;
            L.base_radius = dd == 0 ? ((lv == 0 && nl > 1) ? 0 : 10) : (dd < 0 ? -dd : dd);
        }
        if (L.smallest) {
            L.bw = o.block_w >> 1; L.bh = o.block_h >> 1; L.pxoff = o.block_w >> 2; L.pyoff = o.block_h >> 2;
        } else {
            L.bw = o.block_w; L.bh = o.block_h; L.pxoff = 0; L.pyoff = 0;
        }
        L.tl = ((L.bw + 3) / 4) * ((L.bh + 3) / 4);
        const int cw = L.bw / 2, ch = L.bh / 2;
        L.tc = cw > 0 ? ((cw + 3) / 4) * (((cw > ch ? cw : ch) + 3) / 4) : 0;
        const int64_t cells = (int64_t)L.gw * L.gh;
        if (cells > max_cells) max_cells = cells;
        const int64_t ol = cells + L.gw + L.gh + 8;
        if (ol > max_order) max_order = ol;
        if (L.tl + L.tc > 96 || L.gw > 65535 || L.gh > 65535) { err = "unsupported block / grid size"; return false; }
    }
    {  // level-0 grid must be at least 2x2: below that the reference indexes field[-1]
        if (P.lv[0].gw < 2 || P.lv[0].gh < 2) { err = "SVAnalyse: frame too small for the block grid"; return false; }
    }
    int32_t bw, bh, ox, oy, gw, gh;
    output_block(o, bw, bh, ox, oy);
    output_grid(o, bw, bh, ox, oy, gw, gh);
    P.out_bw = bw; P.out_bh = bh; P.out_ox = ox; P.out_oy = oy; P.out_gw = gw; P.out_gh = gh;
    P.has_refine = o.has_refine_thsad;
    if (P.has_refine) { err = "refine (recalculate) pass is not available on the device path yet"; return false; }
    {  // rescale_scores denominators (:2716-2721)
        double f = sqrt((double)o.width * (double)o.width + (double)o.height * (double)o.height);
        int32_t diag = f != f ? 0 : (f >= 2147483647.0 ? INT32_MAX : (int32_t)f);
        if (diag < 0) diag = 0;
        int64_t den = (int64_t)diag * (bw > 1 ? bw : 1);
        if (den > INT32_MAX) den = INT32_MAX;
        P.rescale_denom = den > 1 ? (int32_t)den : 1;
    }
    P.payload_len = (int64_t)payload_len(o);
    int32_t hdr[16];
    vdata_header(o, hdr);
    // payload words: 16, 0xA0, flags, bw, bh, pel, levels, 0, w, h, ox, oy, gw, gh, selector, delta
    P.header[0] = 16; P.header[1] = 0xA0; P.header[2] = hdr[1]; P.header[3] = bw; P.header[4] = bh;
    P.header[5] = o.pel; P.header[6] = hdr[5]; P.header[7] = 0; P.header[8] = o.width; P.header[9] = o.height;
    P.header[10] = ox; P.header[11] = oy; P.header[12] = gw; P.header[13] = gh; P.header[14] = o.selector;
    P.header[15] = o.delta;
    if ((int64_t)gw * gh != (int64_t)P.lv[0].gw * P.lv[0].gh) { err = "output grid differs from the level-0 grid"; return false; }
    // scratch layout per pair
    int64_t np2 = 1;
    while (np2 < max_cells) np2 <<= 1;
    P.max_cells = max_cells;
    P.max_order = max_order;
    int64_t off = 0;
    auto take = [&](int64_t bytes) { int64_t o_ = off; off += (bytes + 255) & ~(int64_t)255; return o_; };
    for (int dd = 0; dd < 2; dd++) {
        P.off_field[dd] = take(max_cells * 8);
        P.off_next[dd] = take(max_cells * 8);
        P.off_proj[dd][0] = take(max_cells * 8);
        P.off_proj[dd][1] = take(max_cells * 8);
        P.off_order[dd] = take(max_order * 4);
        P.off_order2[dd] = take(max_order * 4);
        P.off_pos[dd] = take(max_cells * 4);
        P.off_keys[dd] = take(np2 * 8 > max_order * 4 ? np2 * 8 : max_order * 4);
        P.off_hist[dd] = take(65536 * 4);
        P.off_seen[dd] = take(max_cells);
        P.off_out[dd] = take(max_cells * 2);
    }
    P.scratch_per_pair = off;
    return true;
}

}  // namespace svpf
