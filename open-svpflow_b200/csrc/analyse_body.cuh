// analyse_body.cuh -- hierarchical block search (Analyse) on sm_100a.
//
// Included by one translation unit per launch variant (analyse_nt128.cu, analyse_nt64.cu,
// analyse_nt32.cu, analyse_nt128b3.cu, analyse_nt64b6.cu): SVPF_NT = threads per search
// direction, SVPF_MINB = resident CTAs per SM the register budget is cut for (2, 4, 8: 128
// registers per thread; 3, 6: 80), SVPF_VARIANT = the variant's namespace. Each variant
// exports a plain launcher (one CTA per pair; in the look-ahead shapes, by default, the pair
// kernel runs the coarser levels, a cooperative level-0 kernel with one CTA per warp walks
// level 0 across the SMs and a finish kernel packs the payloads) and a persistent batch
// launcher (CTAs drain a device work queue of frame pairs from many clips).
//
// Restates crates/svpflow1/src/analyse_search.rs:68-2811 for the GPU:
//   * one CTA per frame pair; its two halves (NT threads each) run the forward search
//     (current -> reference) and the backward search (reference -> current). They meet
//     at a CTA barrier once per level: the forward search of a level needs the
//     backward field of the level above projected onto it, and vice versa (:128-191).
//   * inside a level the blocks run in the reference's serial order (serpentine at
//     level 0, score-sorted at coarser levels, :302-419): each block takes already
//     searched neighbours as candidates, so the order is a true dependency chain and
//     its latency is what the design minimises. Every thread of a half holds the same
//     block state and takes the same decisions, so a search step costs one barrier.
//   * every step of a block's search is a batch of candidate vectors whose positions are
//     known before any is evaluated (special candidates; the UMH cross + hexagons; an
//     exhaustive square; a hexagon step; an expanding ring). A candidate is evaluated by
//     a group of G lanes of one warp, one 4x4 tile per lane (SATD, SAD or pixel sums),
//     reduced with shuffles; each warp keeps the first candidate of minimal cost and
//     the half combines its warps after the step's barrier. First-minimum equals the
//     reference's sequential `if cost < best.cost` scan (:1122-1155) whenever
//     cost >= motion penalty, i.e. pnew >= -256; below that the step replays the
//     sequential scan over each round's costs.
//   * a candidate whose block and reference block lie inside their planes takes the fast
//     path (word loads, packed byte ops); any other candidate takes the reference's own
//     read path (edge-shifted, clamped, masked; :1638-2351) through cand_setup, which
//     keeps the reference's wrapping index arithmetic.
//
// Integer/indexing work: no tensor cores. 8-bit SATD runs in f16x2 on values that halves hold
// exactly (see satd_rows_h); the two f64 formulas (adapt_lambda, exact_lambda) are IEEE-exact
// (exact_lambda is host-precomputed).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "svpf_device.h"

#if !defined(SVPF_NT) || !defined(SVPF_MINB) || !defined(SVPF_VARIANT)
#error "define SVPF_NT, SVPF_MINB and SVPF_VARIANT before including analyse_body.cuh"
#endif
// SVPF_LOOKAHEAD: the shape runs the look-ahead (search_level_spec) when the parameter block asks
// for it. Only the 128-thread shapes with two CTAs per SM (128 registers) do: there it measured
// faster (the 1080p clip: 125.2 -> 134.3 pairs/s); with three CTAs per SM at 80 registers the
// independent warps' instruction fetches cost more than the overlap gains (297 pairs at 960x540:
// 593 -> 692 ms), so the other shapes keep the serial order.
#ifndef SVPF_LOOKAHEAD
#define SVPF_LOOKAHEAD 0
#endif

namespace svpf {
namespace SVPF_VARIANT {

namespace {

#ifdef SVPF_PX16
typedef uint16_t px_t;             // this project's 10-bit extension (no reference behaviour)
constexpr unsigned PX_MID = 512;   // chroma default of the clamped read paths
constexpr unsigned DC_SHIFT = 2;   // the payload's block luma byte is mean >> 2
#else
typedef uint8_t px_t;
constexpr unsigned PX_MID = 128;
constexpr unsigned DC_SHIFT = 0;
#endif
constexpr int NT = SVPF_NT;        // threads per search direction
static_assert(NT == 32 || NT == 64 || NT == 128, "threads per direction");
constexpr int NW = NT / 32;
static_assert(NW <= 4, "the look-ahead keeps at most NW - 1 = 3 deferred seeds per block");
constexpr int NGMAX = NW * 32;     // candidate groups of a direction when a group is one lane
constexpr int MAXSLOT = 16;        // special-candidate slots of a block
constexpr int MW = 4;              // validity mask words per chunk of a search step: 128 candidates

enum : uint8_t { LM_DIRECT = 1, LM_SATD_MASK = 2, LM_SAD_BREAK = 3, LM_EDGE = 4, LM_DC = 5 };
enum : uint8_t { CM_NONE = 0, CM_DIRECT = 1, CM_SAD_BREAK = 3, CM_EDGE = 4 };
enum : int { BK_EXH = 1, BK_UMH, BK_HEX6, BK_HEX3, BK_RING };

constexpr int ST_PANIC = 1;    // status bit: the reference indexes out of range here (it would panic)
constexpr int ST_TIMEOUT = 4;  // status bit: a bounded wait inside the kernel ran out (internal error)
// A wait on another warp's commit gives up after this many SM cycles (about 0.5 s at 1.9 GHz;
// a level-0 block takes well under a millisecond). After one wait of a direction has given
// up, its other waits return at once, so a failure costs one bound, not one per block.
constexpr long long kWaitCycles = 1000000000LL;

struct Cand {
    int64_t l_sbase, l_rbase, c_sbase, c_rbase;  // flat bases of the direct read paths
    int32_t l_sx, l_sy, l_rx, l_ry;              // origins of the clamped / masked paths
    int32_t c_sx, c_sy, c_rx, c_ry;
    int32_t l_srow, l_rrow, c_srow, c_rrow;      // first row of the source / reference sub-plane
    int32_t c_rows;                              // chroma rows covered (n x n for square SATD)
    uint8_t lmode, cmode, lsatd, csatd;
};

// Shared state of one search direction. A block is searched by a group of warps: the whole
// direction (coarser levels), or one warp (level 0 with look-ahead, one block per warp in
// flight). Per-warp entries are indexed by the warp's place in the direction; a group's
// entries are those of its first warp (Ctx::wbase). W: the warps it holds state for (the
// direction's, or one for a CTA of the level-0 kernel).
template <int W>
struct DirShT {
    // Groups that stage a block's source at once: one per warp with the look-ahead, else one per
    // direction (shared memory not used for staging is L1 cache for the rest).
    static constexpr int kSrc = (SVPF_LOOKAHEAD && W > 1) ? W : 1;
    long long K[2][W];                    // per-warp best (cost, index, sad) of a step, double-buffered
    int I[2][W];
    unsigned S[2][W];
    unsigned slotL[W][2][MAXSLOT];        // per group: special-candidate results (exact_sad values)
    long long rk[2][W * 32], rm[2][W * 32];  // exact sequential scan: per-group cost, motion
    unsigned rs[2][W * 32];
    int ri[2][W * 32];
    unsigned char rv[2][W * 32];
    int committed;                        // look-ahead: blocks of the level committed so far (in order)
    int late_;                            // look-ahead: a hand-over wait gave up
    int unsafe_;                          // look-ahead: the level has an input the reference panics on
    int bad_count;                        // look-ahead: bad-SAD blocks committed so far (:605)
    int gx, gy;           // global predictor (doubled) for the next level
    int order_len;
    int abort_;
    // Per group: the block's source pixels, 4 per entry: luma (bw/4 x bh), then U and V
    // (cw/4 x crows). A plane searched with SATD holds biased f16 pairs (8-bit samples; see
    // satd_rows_h) or 16-bit pairs (x = pixels 0,1; y = pixels 2,3), a SAD plane the packed word in x.
    uint2 srcp[kSrc][384];
    int2 clist[W][32 * MW];  // per warp: the step's candidates passing the cuts, in order (mv, index)
    int2 seedv[W][8];        // look-ahead, per group: the block's seeds evaluated at once (vector) ...
    int seedq[W][8];         // ... and their places among the block's processed neighbours;
    long long defc[W][3];    // the deferred seeds' cells (at most NW - 1 = 3) ...
    int defq[W][3];          // ... and places
    long long r64[W][3];
    int r32[W][2];
};
using DirSh = DirShT<NW>;  // a search direction of the pair kernels
using WarpSh = DirShT<1>;  // a CTA (one warp) of the level-0 kernel

struct Planes {
    const px_t *y, *u, *v;
};

struct Geo {  // per level
    int lw, lh, clw, clh;
    int64_t ys, cs, ylen, clen;
    int ys32, cs32;   // the strides again, for 32-bit offsets (planes are below 2^30 bytes)
};

// Named barrier of one search direction (ids 1 and 2; 0 is __syncthreads). Immediate ids,
// so the kernel reserves three barriers, not all sixteen (barriers bound CTAs per SM).
__device__ __forceinline__ void dbar(int d) {
    if (d) asm volatile("bar.sync 2, %0;" ::"n"(NT) : "memory");
    else asm volatile("bar.sync 1, %0;" ::"n"(NT) : "memory");
}
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
__device__ __forceinline__ unsigned rd(const px_t *p, int64_t len, int64_t i, unsigned dflt) {
    return (i >= 0 && i < len) ? (unsigned)__ldg(p + i) : dflt;
}
__device__ __forceinline__ long long pen(int pnew, unsigned x) { return (long long)x + (((long long)pnew * (long long)x) >> 8); }
// (lambda * |pred - mv|^2) >> 8; vectors are below 2^16 in magnitude, so the differences
// fit 32 bits and the squares are single widening multiplies
__device__ __forceinline__ long long motion_penalty(int lambda, int px_, int py_, int mx, int my) {
    const int dx = px_ - mx, dy = py_ - my;
    return ((long long)lambda * ((long long)dx * dx + (long long)dy * dy)) >> 8;
}

// hadamard4_satd, analyse_search.rs:2681-2702: rows, then columns; the last column
// stage and its absolute values use |a+b| + |a-b| = 2 max(|a|, |b|).
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
        s += max(abs(s0), abs(s2)) + max(abs(s1), abs(s3));
    }
    return (unsigned)(2 * s);
}

// -------------------------------------------------------------------------------------------
// Candidate set-up on the reference's read paths (any candidate; the general path).
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

// One 4x4 tile of one chroma plane of a candidate on the general path.
__device__ unsigned chroma_tile1(const Cand &c, const px_t *sp, const px_t *rp, const Geo &G, int cw, int tile) {
    if (c.cmode == CM_NONE) return 0;
    const int txn = (cw + 3) >> 2;
    const int ty = tile / txn, tx = tile - ty * txn;
    const int r0 = ty * 4, c0 = tx * 4;
    if (r0 >= c.c_rows || c0 >= cw) return 0;
    const int hh = imin(4, c.c_rows - r0), ww = imin(4, cw - c0);
    const int64_t cs = G.cs, clen = G.clen;
    const int clw = G.clw, clh = G.clh;
    int d[16];
#pragma unroll
    for (int i = 0; i < 16; i++) d[i] = 0;
    if (c.cmode == CM_DIRECT) {
#pragma unroll
        for (int r = 0; r < 4; r++)
#pragma unroll
            for (int q = 0; q < 4; q++)
                if (r < hh && q < ww)
                    d[r * 4 + q] = (int)rd(sp, clen, c.c_sbase + (int64_t)(r0 + r) * cs + c0 + q, 0) -
                                   (int)rd(rp, clen, c.c_rbase + (int64_t)(r0 + r) * cs + c0 + q, 0);
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
                    d[r * 4 + q] = (int)rd(sp, clen, ((int64_t)c.c_srow + sy) * cs + sx, PX_MID) -
                                   (int)rd(rp, clen, ((int64_t)c.c_rrow + ry) * cs + rx, PX_MID);
                }
            }
        }
    } else {  // CM_EDGE
        const int mh = imax(clh - 1, 0), mw = imax(clw - 1, 0);
        const unsigned dflt = c.csatd ? 0u : PX_MID;
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const int sy = iclamp(c.c_sy + r0 + r, 0, mh), ry = iclamp(c.c_ry + r0 + r, 0, mh);
#pragma unroll
            for (int q = 0; q < 4; q++)
                if (r < hh && q < ww) {
                    const int sx = iclamp(c.c_sx + c0 + q, 0, mw), rx = iclamp(c.c_rx + c0 + q, 0, mw);
                    d[r * 4 + q] = (int)rd(sp, clen, ((int64_t)c.c_srow + sy) * cs + sx, dflt) -
                                   (int)rd(rp, clen, ((int64_t)c.c_rrow + ry) * cs + rx, dflt);
                }
        }
    }
    if (c.csatd) return hadamard4(d);
    unsigned s = 0;
#pragma unroll
    for (int i = 0; i < 16; i++) s += (unsigned)abs(d[i]);
    return s;
}

// -------------------------------------------------------------------------------------------
// Fast path: candidates whose source and reference blocks lie inside their planes.
// Samples are read as 32-bit words from 4-byte aligned addresses and funnel-shifted; the
// caller guarantees 8 readable samples after the first sample of every row (see fast_setup).
//
// SATD runs in packed halfwords: a row's four sample differences are two halfword pairs
// (samples 0,1 and 2,3); the horizontal 4-point transform runs inside the pairs, the vertical
// one across the rows, and the last vertical stage with its absolute values is
// |a+b| + |a-b| = 2 max(|a|, |b|), as in hadamard4. Every intermediate fits a signed halfword
// (|value| <= 8 * max sample) and the four-row sum an unsigned one.
__device__ __forceinline__ unsigned satd_rows(const uint32_t d01[4], const uint32_t d23[4]) {
    uint32_t h0[4], h1[4];
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const uint32_t c = __vadd2(d01[r], d23[r]), e = __vsub2(d01[r], d23[r]);
        const uint32_t p = __byte_perm(c, e, 0x5410), q = __byte_perm(c, e, 0x7632);
        h0[r] = __vadd2(p, q);
        h1[r] = __vsub2(p, q);
    }
    uint32_t acc = 0;
#pragma unroll
    for (int k = 0; k < 2; k++) {
        const uint32_t *h = k ? h1 : h0;
        const uint32_t a0 = __vadd2(h[0], h[1]), a1 = __vsub2(h[0], h[1]);
        const uint32_t a2 = __vadd2(h[2], h[3]), a3 = __vsub2(h[2], h[3]);
        acc = __vadd2(acc, __vmaxu2(__vabs2(a0), __vabs2(a2)));
        acc = __vadd2(acc, __vmaxu2(__vabs2(a1), __vabs2(a3)));
    }
    return 2u * ((acc & 0xFFFFu) + (acc >> 16));
}
__device__ __forceinline__ uint32_t pairs_lo(uint32_t w) { return __byte_perm(w, 0u, 0x4140); }  // bytes 0, 1
__device__ __forceinline__ uint32_t pairs_hi(uint32_t w) { return __byte_perm(w, 0u, 0x4342); }  // bytes 2, 3

#ifndef SVPF_PX16
// 8-bit SATD runs in f16x2 instead: a sample s becomes the half 1024 + s (exponent of 1024,
// s in the mantissa: one byte permute), so a difference of two samples is exact, and so is
// every later value (integers of magnitude <= 8 * 255 = 2040 <= 2048, where halves are
// exact). The four-row sums go to f32. Same arithmetic as satd_rows, fewer instructions
// (the f16x2 add / sub / max are single instructions; |x| clears the sign bits).
__device__ __forceinline__ uint32_t bias_lo(uint32_t w) { return __byte_perm(w, 0x64646464u, 0x4140); }
__device__ __forceinline__ uint32_t bias_hi(uint32_t w) { return __byte_perm(w, 0x64646464u, 0x4342); }
__device__ __forceinline__ uint32_t h2add(uint32_t a, uint32_t b) {
    uint32_t d;
    asm("add.rn.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
}
__device__ __forceinline__ uint32_t h2sub(uint32_t a, uint32_t b) {
    uint32_t d;
    asm("sub.rn.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
}
__device__ __forceinline__ uint32_t h2max(uint32_t a, uint32_t b) {
    uint32_t d;
    asm("max.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
}
__device__ __forceinline__ uint32_t h2abs(uint32_t a) { return a & 0x7FFF7FFFu; }
// acc + both halves of h, in f32 (sm_100 mixed-precision add)
__device__ __forceinline__ float f32_add_h2(float acc, uint32_t h) {
    asm("{.reg .b16 l, h; mov.b32 {l, h}, %1; add.rn.f32.f16 %0, l, %0; add.rn.f32.f16 %0, h, %0;}"
        : "+f"(acc) : "r"(h));
    return acc;
}
// d01 / d23: the rows' differences as f16 pairs (samples 0,1 and 2,3)
__device__ __forceinline__ unsigned satd_rows_h(const uint32_t d01[4], const uint32_t d23[4]) {
    uint32_t h0[4], h1[4];
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const uint32_t c = h2add(d01[r], d23[r]), e = h2sub(d01[r], d23[r]);
        const uint32_t p = __byte_perm(c, e, 0x5410), q = __byte_perm(c, e, 0x7632);
        h0[r] = h2add(p, q);
        h1[r] = h2sub(p, q);
    }
    float acc = 0.f;
#pragma unroll
    for (int k = 0; k < 2; k++) {
        const uint32_t *h = k ? h1 : h0;
        const uint32_t a0 = h2add(h[0], h[1]), a1 = h2sub(h[0], h[1]);
        const uint32_t a2 = h2add(h[2], h[3]), a3 = h2sub(h[2], h[3]);
        acc = f32_add_h2(acc, h2max(h2abs(a0), h2abs(a2)));
        acc = f32_add_h2(acc, h2max(h2abs(a1), h2abs(a3)));
    }
    return 2u * (unsigned)acc;
}
__device__ __forceinline__ uint32_t ld4u(const uint8_t *p) {
    const uintptr_t a = (uintptr_t)p;
    const uint32_t *q = reinterpret_cast<const uint32_t *>(a & ~(uintptr_t)3);
    return __funnelshift_r(__ldg(q), __ldg(q + 1), (unsigned)(a & 3) * 8u);
}
// four samples as biased f16 pairs
__device__ __forceinline__ uint2 ld4h(const px_t *p) {
    const uint32_t w = ld4u(p);
    return make_uint2(bias_lo(w), bias_hi(w));
}
// The staged entry of 4 source samples for a plane searched with SATD (biased f16 pairs) or
// SAD (the packed word).
__device__ __forceinline__ uint2 stage4(const px_t *p, bool satd) {
    const uint32_t w = ld4u(p);
    return satd ? make_uint2(bias_lo(w), bias_hi(w)) : make_uint2(w, 0u);
}
__device__ __forceinline__ unsigned sad4(uint2 staged, const px_t *rp) {
    return __dp4a(__vabsdiffu4(staged.x, ld4u(rp)), 0x01010101u, 0u);
}
__device__ __forceinline__ unsigned sad4g(const px_t *sp, const px_t *rp) {
    return __dp4a(__vabsdiffu4(ld4u(sp), ld4u(rp)), 0x01010101u, 0u);
}
__device__ __forceinline__ unsigned sum4(const px_t *p) { return __dp4a(ld4u(p), 0x01010101u, 0u); }
#else
// four 16-bit samples (2-byte aligned): three aligned words funnel-shifted into two pairs
__device__ __forceinline__ uint2 ld4p(const px_t *p) {
    const uintptr_t a = (uintptr_t)p;
    const uint32_t *q = reinterpret_cast<const uint32_t *>(a & ~(uintptr_t)3);
    const unsigned sh = (unsigned)(a & 3) * 8u;
    const uint32_t w0 = __ldg(q), w1 = __ldg(q + 1), w2 = __ldg(q + 2);
    return make_uint2(__funnelshift_r(w0, w1, sh), __funnelshift_r(w1, w2, sh));
}
__device__ __forceinline__ uint2 stage4(const px_t *p, bool) { return ld4p(p); }
__device__ __forceinline__ unsigned sad4(uint2 staged, const px_t *rp) {
    const uint2 r = ld4p(rp);
    return __vsadu2(staged.x, r.x) + __vsadu2(staged.y, r.y);
}
__device__ __forceinline__ unsigned sad4g(const px_t *sp, const px_t *rp) { return sad4(ld4p(sp), rp); }
__device__ __forceinline__ unsigned sum4(const px_t *p) {
    const uint2 w = ld4p(p);
    return (w.x & 0xFFFFu) + (w.x >> 16) + (w.y & 0xFFFFu) + (w.y >> 16);
}
#endif

// tiles with both blocks in global memory (special candidates)
__device__ __forceinline__ unsigned tile_satd(const px_t *sp, const px_t *rp, int st) {
    uint32_t d01[4], d23[4];
#ifndef SVPF_PX16
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const uint2 a = ld4h(sp + r * st), b = ld4h(rp + r * st);
        d01[r] = h2sub(a.x, b.x);
        d23[r] = h2sub(a.y, b.y);
    }
    return satd_rows_h(d01, d23);
#else
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const uint2 a = ld4p(sp + r * st), b = ld4p(rp + r * st);
        d01[r] = __vsub2(a.x, b.x);
        d23[r] = __vsub2(a.y, b.y);
    }
    return satd_rows(d01, d23);
#endif
}
__device__ __forceinline__ unsigned tile_sad(const px_t *sp, const px_t *rp, int st) {
    unsigned s = 0;
#pragma unroll
    for (int r = 0; r < 4; r++) s += sad4g(sp + r * st, rp + r * st);
    return s;
}
// tiles over the staged source (see DirSh::srcp)
__device__ __forceinline__ unsigned tile_satd_p(const uint2 *sp, int spp, const px_t *rp, int st) {
    uint32_t d01[4], d23[4];
#ifndef SVPF_PX16
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const uint2 a = sp[r * spp], b = ld4h(rp + r * st);
        d01[r] = h2sub(a.x, b.x);
        d23[r] = h2sub(a.y, b.y);
    }
    return satd_rows_h(d01, d23);
#else
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const uint2 a = sp[r * spp], b = ld4p(rp + r * st);
        d01[r] = __vsub2(a.x, b.x);
        d23[r] = __vsub2(a.y, b.y);
    }
    return satd_rows(d01, d23);
#endif
}
__device__ __forceinline__ unsigned tile_sad_p(const uint2 *sp, int spp, const px_t *rp, int st) {
    unsigned s = 0;
#pragma unroll
    for (int r = 0; r < 4; r++) s += sad4(sp[r * spp], rp + r * st);
    return s;
}
__device__ __forceinline__ unsigned tile_sum(const px_t *sp, int st) {
    unsigned s = 0;
#pragma unroll
    for (int r = 0; r < 4; r++) s += sum4(sp + r * st);
    return s;
}

// -------------------------------------------------------------------------------------------
// candidate generators (the reference's loop orders)
__constant__ int2 c_hex2[8] = {{-1, -2}, {-2, 0}, {-1, 2}, {1, 2}, {2, 0}, {1, -2}, {-1, -2}, {-2, 0}};  // :889-898
__constant__ int c_mod6m1[8] = {5, 0, 1, 2, 3, 4, 5, 0};
__constant__ int2 c_hex4[16] = {{-4, 2}, {-4, 1}, {-4, 0}, {-4, -1}, {-4, -2}, {4, -2}, {4, -1}, {4, 0},
                                {4, 1},  {4, 2},  {2, 3},  {0, 4},   {-2, 3},  {-2, -3}, {0, -4}, {2, -3}};  // :1075-1092

struct Gen {
    int kind, cx, cy, r, step, odir, n;
};
__device__ __forceinline__ int ring_m(int r, int step) { return 2 * r > step ? (2 * r - 1) / step : 0; }
__device__ __forceinline__ Gen make_gen(int kind, int cx, int cy, int r, int step, int odir) {
    Gen g{kind, cx, cy, r, step, odir, 0};
    switch (kind) {
    case BK_EXH: g.n = (2 * r + 1) * (2 * r + 1); break;
    case BK_UMH: g.n = 4 * (r / 2 > 0 ? r / 2 : 0) + 16 * imax(r / 4, 1); break;
    case BK_HEX6: g.n = 6; break;
    case BK_HEX3: g.n = 3; break;
    case BK_RING: g.n = 4 * ring_m(r, step) + 4; break;
    }
    return g;
}
__device__ int2 gen_mv(const Gen &g, int i) {
    const int cx = g.cx, cy = g.cy, r = g.r;
    switch (g.kind) {
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
    case BK_HEX3: { int2 h = c_hex2[g.odir + i]; return make_int2(cx + h.x, cy + h.y); }
    case BK_RING: {  // exact_expanding, :849-885
        const int step = g.step, m = ring_m(r, step);
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

// -------------------------------------------------------------------------------------------
struct Ctx {
    const AnalyseParams *P;
    const LevelInfo *L;
    Geo G;
    Planes S, R;
    int level, d, tid, satd, pel;
    int nw, wbase;   // warps of the group searching the block, and its first warp in the direction;
                     // tid is the thread's index in that group
    int grp_lanes;   // G: lanes per candidate (power of two)
    int pnew;        // new-candidate penalty of the current search (opts.pnew; pnew / factor in the refine pass)
    int tl, tcp;     // 4x4 luma tiles, 4x4 tiles per chroma plane of one candidate
};

// Barrier of the group searching a block: the direction's named barrier, or the warp.
__device__ __forceinline__ void gsync(const Ctx &x) {
    if (x.nw == 1) __syncwarp();
    else dbar(x.d);
}

// Per-block constants, identical in every thread of a direction.
struct BlkC {
    int px, py, bw, bh, px2, py2;
    int bnd0, bnd1, bnd2, bnd3, ubx, uby;  // mv_bounds; ub = bound above which the edge shift starts
    int chroma, satd_mode, fastable, fast_src, cfast_src, dc_fast;
    int cw, ch, crows, cpx, cpy, tilesx, ctilesx;
    int lgtx, lgctx;                       // log2 of tilesx / ctilesx (block sizes are powers of two)
    int fx0, fx1, fy0, fy1;                // vectors taking the fast path lie in this box (inclusive) ...
    int lbase, llim, cbase, clim;          // ... and have lref <= llim, cref <= clim (offsets from these bases)
    int64_t lsrc, csrc, dsrc;              // flat index of the source block (luma, chroma, luma at (px, py))
};

__device__ __forceinline__ void make_blk(const Ctx &x, int px, int py, bool chroma, BlkC &b) {
    const LevelInfo &L = *x.L;
    const Geo &G = x.G;
    const int bw = L.bw, bh = L.bh, pel = imax(x.pel, 1);
    b.px = px; b.py = py; b.bw = bw; b.bh = bh;
    b.px2 = px - (x.level > 0 && px + bw >= G.lw);
    b.py2 = py - (x.level > 0 && py + bh >= G.lh);
    b.bnd0 = -pel * px; b.bnd1 = -pel * py;
    b.bnd2 = pel * (G.lw - px - bw) + 1; b.bnd3 = pel * (G.lh - py - bh) + 1;
    b.ubx = b.bnd2 > b.bnd0 ? b.bnd2 : 0x7FFFFFFF;
    b.uby = b.bnd3 > b.bnd1 ? b.bnd3 : 0x7FFFFFFF;
    b.chroma = chroma;
    b.satd_mode = x.satd && is_blk(bw) && is_blk(bh) && bw == bh;
    b.fastable = bw > 0 && bh > 0 && (bw & 3) == 0 && (bh & 3) == 0;
    b.tilesx = bw >> 2;
    b.lgtx = 31 - __clz(imax(b.tilesx, 1));
    b.lsrc = ((int64_t)L.y_off + b.py2) * G.ys + b.px2;
    b.fast_src = b.fastable && b.px2 >= 0 && b.py2 >= 0 && b.px2 + bw <= G.lw && b.py2 + bh <= G.lh &&
                 b.lsrc + (int64_t)(bh - 1) * G.ys + bw + 8 <= G.ylen;
    b.dsrc = ((int64_t)L.y_off + py) * G.ys + px;
    b.dc_fast = b.fastable && px >= 0 && py >= 0 && px + bw <= G.lw && py + bh <= G.lh &&
                b.dsrc + (int64_t)(bh - 1) * G.ys + bw + 8 <= G.ylen;
    b.cw = bw / 2; b.ch = bh / 2;
    b.crows = x.satd ? b.cw : b.ch;
    b.ctilesx = (b.cw + 3) >> 2;
    b.lgctx = 31 - __clz(imax(b.ctilesx, 1));
    b.cpx = px / 2; b.cpy = py / 2;
    b.csrc = ((int64_t)L.c_off + b.cpy) * G.cs + b.cpx;
    b.cfast_src = (b.cw == 4 || b.cw == 8 || b.cw == 16) && b.ch >= 4 && (b.ch & 3) == 0 && px >= 0 && py >= 0 &&
                  b.cpx + b.cw <= G.clw && b.cpy + b.ch <= G.clh &&
                  b.csrc + (int64_t)(b.crows - 1) * G.cs + b.cw + 8 <= G.clen;
    // the fast-path box: no edge shift, reference block inside the level (luma, and chroma when
    // it is evaluated); with l0sub the luma offset is mv >> 1 and the chroma one mv >> 2
    const bool l0sub = x.level == 0 && pel >= 2;
    const int ls = l0sub ? 1 : 0, cshift = l0sub ? 2 : 1;
    b.fx0 = imax(b.bnd0, (-b.px2) * (1 << ls));
    b.fx1 = imin(b.ubx - 1, (G.lw - bw - b.px2) * (1 << ls) + (1 << ls) - 1);
    b.fy0 = imax(b.bnd1, (-b.py2) * (1 << ls));
    b.fy1 = imin(b.uby - 1, (G.lh - bh - b.py2) * (1 << ls) + (1 << ls) - 1);
    if (b.chroma && b.cw >= 4 && b.ch >= 4) {
        b.fx0 = imax(b.fx0, (-b.cpx) * (1 << cshift));
        b.fx1 = imin(b.fx1, (G.clw - b.cw - b.cpx) * (1 << cshift) + (1 << cshift) - 1);
        b.fy0 = imax(b.fy0, (-b.cpy) * (1 << cshift));
        b.fy1 = imin(b.fy1, (G.clh - b.ch - b.cpy) * (1 << cshift) + (1 << cshift) - 1);
        if (!b.cfast_src) b.fx1 = b.fx0 - 1;
    }
    if (!b.fast_src) b.fx1 = b.fx0 - 1;  // empty box
    b.lbase = (int)L.y_off * G.ys32;
    b.llim = (int)G.ylen - (bh - 1) * G.ys32 - bw - 8;
    b.cbase = (int)L.c_off * G.cs32;
    b.clim = (int)G.clen - (b.crows - 1) * G.cs32 - b.cw - 8;
}

// Does (block, mv) take the fast path? If so, the flat indices of its reference blocks.
// It does when the reference takes its direct reads for both luma and chroma: no edge
// shift, the luma block and the reference block inside the level, the chroma blocks too.
__device__ __forceinline__ bool fast_setup(const Ctx &x, const BlkC &b, int mvx, int mvy, int &lref, int &cref) {
    if (mvx < b.fx0 || mvx > b.fx1 || mvy < b.fy0 || mvy > b.fy1) return false;
    const int pel = imax(x.pel, 1);
    const bool l0sub = x.level == 0 && pel >= 2;
    const int sub = l0sub ? (mvy & 1) * pel + (mvx & 1) : 0;
    const int mx = l0sub ? mvx >> 1 : mvx, my = l0sub ? mvy >> 1 : mvy;
    lref = b.lbase + (sub * x.G.lh + b.py2 + my) * x.G.ys32 + b.px2 + mx;
    if (lref > b.llim) return false;
    cref = 0;
    if (b.chroma && b.cw >= 4 && b.ch >= 4) {
        const int mcx = l0sub ? mvx >> 2 : mvx >> 1, mcy = l0sub ? mvy >> 2 : mvy >> 1;
        cref = b.cbase + ((l0sub ? sub * x.G.clh : 0) + b.cpy + mcy) * x.G.cs32 + b.cpx + mcx;
        if (cref > b.clim) return false;
    }
    return true;
}

struct Res {
    unsigned L, U, V;
    int lsatd, cmode, csatd;
};

// The general path for one lane: the reference's own read path through cand_setup.
// Arguments by value only, so nothing of the caller's state lives in local memory.
__device__ __noinline__ Res slow_lane(const AnalyseParams *P, const LevelInfo *L, Geo G, Planes S, Planes R, int level,
                                      int px, int py, int bw, int bh, int mvx, int mvy, bool chroma, int satd, int pel,
                                      bool dc, int sub, int Gl, int TL, int TCp) {
    Res r{0, 0, 0, 0, 0, 0};
    Cand c;
    cand_setup(c, *P, *L, G, level, px, py, bw, bh, mvx, mvy, chroma, satd, pel, dc);
    r.lsatd = c.lsatd; r.cmode = c.cmode; r.csatd = c.csatd;
    const int T = TL + (chroma ? 2 * TCp : 0);
    for (int t = sub; t < T; t += Gl) {
        if (t < TL) r.L += luma_tile(c, S, R, G, bw, bh, t);
        else if (c.cmode != CM_NONE) {
            int ct = t - TL;
            const int pl = ct >= TCp;
            ct -= pl * TCp;
            const unsigned v = chroma_tile1(c, pl ? S.v : S.u, pl ? R.v : R.u, G, bw / 2, ct);
            if (pl) r.V += v; else r.U += v;
        }
    }
    return r;
}


// Lanes per candidate for a step of n candidates: the widest power-of-two group (at most a
// warp, at least the level's G) that still puts every candidate in one round. Small steps
// (a hexagon, a ring, the special candidates) then finish in fewer tiles per lane.
__device__ __forceinline__ int step_lanes(int G, int n, int nw) {
    while (G < 32 && nw * (16 / G) >= n) G <<= 1;
    return G;
}

// Work of one lane (`sub` of G) on one candidate: its share of the 4x4 tiles.
// kind 0: block at (b.px, b.py); 1: the same mv on the block at (px, py) (general path);
// 2: the block's luma pixel sum (block_luma_dc).
__device__ __forceinline__ Res eval_lane(const Ctx &x, const BlkC &b, int kind, int px, int py, int mvx, int mvy,
                                         bool chroma, int sub, int G) {
    const int TL = x.tl, TCp = x.tcp;
    int lref = 0, cref = 0;
    bool fast = false;
    if (kind == 0) fast = fast_setup(x, b, mvx, mvy, lref, cref);
    else if (kind == 2) fast = b.dc_fast;
    if (!fast)
        return slow_lane(x.P, x.L, x.G, x.S, x.R, x.level, kind == 1 ? px : b.px, kind == 1 ? py : b.py, b.bw, b.bh,
                         mvx, mvy, chroma, x.satd, x.pel, kind == 2, sub, G, TL, TCp);
    Res r{0, 0, 0, 0, 0, 0};
    const int T = TL + (chroma ? 2 * TCp : 0);
    const int ys = x.G.ys32, cs = x.G.cs32;
    r.lsatd = kind == 2 ? 0 : b.satd_mode;
    r.cmode = (chroma && b.cw >= 4 && b.ch >= 4) ? CM_DIRECT : CM_NONE;
    r.csatd = x.satd;
    const px_t *sl = x.S.y + (kind == 2 ? b.dsrc : b.lsrc);
#pragma unroll 1
    for (int t = sub; t < T; t += G) {
        if (t < TL) {
            const int ty = t >> b.lgtx, tx = t & (b.tilesx - 1);
            const int o = ty * 4 * ys + tx * 4;
            if (kind == 2) r.L += tile_sum(sl + o, ys);
            else if (r.lsatd) r.L += tile_satd(sl + o, x.R.y + lref + o, ys);
            else r.L += tile_sad(sl + o, x.R.y + lref + o, ys);
        } else if (r.cmode != CM_NONE) {
            int ct = t - TL;
            const int pl = ct >= TCp;
            ct -= pl * TCp;
            const int ty = ct >> b.lgctx, tx = ct & (b.ctilesx - 1);
            if (ty * 4 >= b.crows) continue;
            const int o = ty * 4 * cs + tx * 4;
            const px_t *sp = (pl ? x.S.v : x.S.u) + b.csrc + o, *rp = (pl ? x.R.v : x.R.u) + cref + o;
            const unsigned v = r.csatd ? tile_satd(sp, rp, cs) : tile_sad(sp, rp, cs);
            if (pl) r.V += v; else r.U += v;
        }
    }
    return r;
}

// the three sums of a group of G lanes (independent shuffles, so they overlap)
__device__ __forceinline__ void group_sum3(Res &r, int G) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        if (o < G) {
            r.L += __shfl_xor_sync(0xFFFFFFFFu, r.L, o);
            r.U += __shfl_xor_sync(0xFFFFFFFFu, r.U, o);
            r.V += __shfl_xor_sync(0xFFFFFFFFu, r.V, o);
        }
    }
}
__device__ __forceinline__ void finalize(const Res &r, unsigned &L, unsigned &C) {
    L = r.lsatd ? (r.L >> 1) : r.L;
    if (r.cmode == CM_NONE) C = 0;
    else if (r.csatd) C = sat_mul(sat_add(r.U >> 1, r.V >> 1), 4);
    else C = sat_mul(r.U + r.V, 4);
}

// One search step: candidates g over the block against the running best `best_cost`.
// Every warp computes which candidates pass exact_ok and the motion-penalty cut (a
// ballot bitmask, identical in every warp), then groups take the passing candidates
// in order. On return, identically in every thread: win = accepted candidate or -1,
// and the new best cost / sad when accepted.
template <class SH>
__device__ __forceinline__ void eval_step(const Ctx &x, const BlkC &b, SH &s, int &ph, const Gen &g, int lambda,
                                          int predx, int predy, long long &best_cost, unsigned &best_sad, int &win) {
    const int lane = x.tid & 31, warp = x.tid >> 5, wi = x.wbase + warp;  // wi: the warp's place in the direction
    const bool serial = x.pnew < -256;
    const int pnew = x.pnew;
    long long bk = 0x7FFFFFFFFFFFFFFFLL;
    int bi = 0x7FFFFFFF;
    unsigned bs = 0;
    win = -1;
    const unsigned lt_mask = (1u << lane) - 1u;
    for (int base = 0; base < g.n; base += 32 * MW) {
        int total = 0;
        const long long cut = best_cost;
        // this warp's copy of the passing candidates, in candidate order (every warp
        // computes the same list, so no barrier is needed)
#pragma unroll 1
        for (int w = 0; w < MW; w++) {
            if (base + w * 32 >= g.n) break;  // uniform
            const int i = base + w * 32 + lane;
            bool ok = i < g.n;
            int2 mv = make_int2(0, 0);
            if (ok) {
                mv = gen_mv(g, i);
                ok = mv.x >= b.bnd0 && mv.y >= b.bnd1 && mv.x < b.bnd2 && mv.y < b.bnd3;  // exact_ok
                if (ok) ok = motion_penalty(lambda, predx, predy, mv.x, mv.y) < cut;  // a later candidate faces a lower best
            }
            const unsigned m = __ballot_sync(0xFFFFFFFFu, ok);
            if (ok)  // |mv| <= pel * plane size, so each component fits a halfword
                s.clist[wi][total + __popc(m & lt_mask)] =
                    make_int2((int)(((unsigned)mv.x & 0xFFFFu) | ((unsigned)mv.y << 16)), i);
            total += __popc(m);
        }
        __syncwarp();
        const int G = step_lanes(x.grp_lanes, total, x.nw);
        const int grp = warp * (32 / G) + lane / G, sub = lane & (G - 1), NG = x.nw * (32 / G);
        const int rb = x.wbase * 32;  // the group's entries of the sequential-scan arrays
        for (int r0 = 0; r0 < total; r0 += NG) {
            const int rk = r0 + grp;
            const bool act = rk < total;
            int i = 0;
            int2 mv = make_int2(0, 0);
            if (act) {  // the rk-th passing candidate
                const int2 e = s.clist[wi][rk];
                i = e.y;
                mv = make_int2((int)(short)(e.x & 0xFFFF), e.x >> 16);
            }
            int lref = 0, cref = 0;
            bool fast = false;
            Res r{0, 0, 0, 0, 0, 0};
            long long motion = 0;
            if (act) {
                motion = motion_penalty(lambda, predx, predy, mv.x, mv.y);
                fast = fast_setup(x, b, mv.x, mv.y, lref, cref);
                if (!fast)
                    r = slow_lane(x.P, x.L, x.G, x.S, x.R, x.level, b.px, b.py, b.bw, b.bh, mv.x, mv.y, b.chroma != 0,
                                  x.satd, x.pel, false, sub, G, x.tl, x.tcp);
            }
            // this lane's 4x4 tiles: luma, then U, then V (the source block is staged in shared memory)
            if (act && fast) {
                r.lsatd = b.satd_mode;
                r.cmode = (b.chroma && b.cw >= 4 && b.ch >= 4) ? CM_DIRECT : CM_NONE;
                r.csatd = x.satd;
                const int T = x.tl + (r.cmode != CM_NONE ? 2 * x.tcp : 0);
                const int ys = x.G.ys32, cs = x.G.cs32, nlw = b.tilesx * b.bh;
                const px_t *rl = x.R.y + lref;
                int t = sub;  // luma tiles, then chroma: two loops, no per-tile branch on the plane
#pragma unroll 1
                for (; t < x.tl; t += G) {
                    const int ty = t >> b.lgtx, tx = t & (b.tilesx - 1);
                    const px_t *rp = rl + (ty * 4 * ys + tx * 4);
                    const uint2 *sp = s.srcp[SH::kSrc > 1 ? x.wbase : 0] + ((ty * 4) << b.lgtx) + tx;
                    r.L += b.satd_mode ? tile_satd_p(sp, b.tilesx, rp, ys) : tile_sad_p(sp, b.tilesx, rp, ys);
                }
#pragma unroll 1
                for (; t < T; t += G) {
                    const int ct0 = t - x.tl;
                    const int pl = ct0 >= x.tcp;
                    const int ct = ct0 - pl * x.tcp;
                    const int ty = ct >> b.lgctx, tx = ct & (b.ctilesx - 1);
                    if (ty * 4 >= b.crows) continue;
                    const px_t *rp = (pl ? x.R.v : x.R.u) + cref + (ty * 4 * cs + tx * 4);
                    const uint2 *sp = s.srcp[SH::kSrc > 1 ? x.wbase : 0] + nlw + pl * b.ctilesx * b.crows +
                                      ((ty * 4) << b.lgctx) + tx;
                    const unsigned v = x.satd ? tile_satd_p(sp, b.ctilesx, rp, cs) : tile_sad_p(sp, b.ctilesx, rp, cs);
                    if (pl) r.V += v; else r.U += v;
                }
            }
            group_sum3(r, G);
            long long K = 0x7FFFFFFFFFFFFFFFLL;
            unsigned sad = 0;
            if (act) {
                unsigned L, C;
                finalize(r, L, C);
                if (!b.chroma) C = 0;
                K = motion + pen(pnew, L) + (b.chroma ? pen(pnew, C) : 0LL);  // :1158-1221
                sad = sat_add(L, C);
            }
            if (serial) {  // exact sequential semantics for penalties that can be negative
                if (sub == 0) {
                    s.rk[ph][rb + grp] = K; s.rm[ph][rb + grp] = motion; s.rs[ph][rb + grp] = sad;
                    s.rv[ph][rb + grp] = act; s.ri[ph][rb + grp] = i;
                }
                gsync(x);
                const int m = imin(NG, total - r0);
                for (int j = rb; j < rb + m; j++) {
                    if (s.rm[ph][j] >= best_cost) continue;
                    if (s.rk[ph][j] < best_cost) { best_cost = s.rk[ph][j]; best_sad = s.rs[ph][j]; win = s.ri[ph][j]; }
                }
                ph ^= 1;
            } else if (act && sub == 0 && (K < bk || (K == bk && i < bi))) {
                bk = K; bi = i; bs = sad;
            }
        }
        __syncwarp();  // the next chunk rewrites this warp's list
    }
    if (serial) return;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const long long ok_ = __shfl_xor_sync(0xFFFFFFFFu, bk, o);
        const int oi = __shfl_xor_sync(0xFFFFFFFFu, bi, o);
        const unsigned os = __shfl_xor_sync(0xFFFFFFFFu, bs, o);
        if (ok_ < bk || (ok_ == bk && oi < bi)) { bk = ok_; bi = oi; bs = os; }
    }
    if (x.nw > 1) {  // combine the group's warps (one warp already holds its result in every lane)
        if (lane == 0) { s.K[ph][wi] = bk; s.I[ph][wi] = bi; s.S[ph][wi] = bs; }
        gsync(x);
        bk = s.K[ph][x.wbase]; bi = s.I[ph][x.wbase]; bs = s.S[ph][x.wbase];
        for (int w = x.wbase + 1; w < x.wbase + x.nw; w++) {
            const long long k = s.K[ph][w];
            const int ii = s.I[ph][w];
            if (k < bk || (k == bk && ii < bi)) { bk = k; bi = ii; bs = s.S[ph][w]; }
        }
    }
    ph ^= 1;
    if (bi != 0x7FFFFFFF && bk < best_cost) { best_cost = bk; best_sad = bs; win = bi; }
}

// adapt_lambda, :1555-1564 (f64, IEEE-exact: one add, one division, two products)
__device__ __forceinline__ int adapt_lambda(int nlambda, int lsad, unsigned pred_score) {
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
__device__ __noinline__ unsigned plane_activity(const px_t *data, int64_t len, int64_t stride, int64_t row, int64_t x,
                                                int w, int h, bool satd) {
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

__device__ __forceinline__ int adaptive_radius(int radius, unsigned act) {
    if (act < 2) return 0;
    unsigned a = 255u * act / 150u;
    return ((radius * (int)(a < 255 ? a : 255)) >> 8) + 1;
}
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

// search states of one block (exact_search_block :684-768, exact_refine_search :771-826,
// exact_hex2 :942-1033, exact_umh :1036-1119, bad-SAD expansion :611-672)
enum { S_REFINE, S_HEX_START, S_HEX_ITER, S_HEX_EXIT, S_BAD, S_BAD_RING, S_FINAL_RING, S_STORE };

// The block's source pixels into shared memory (DirSh::srcp) for the fast path.
template <class SH>
__device__ __forceinline__ void stage_source(const Ctx &x, SH &s, const BlkC &b) {
    if (b.fast_src) {
        const int nlw = b.tilesx * b.bh;
        const int nth = x.nw * 32;
        uint2 *sp = s.srcp[SH::kSrc > 1 ? x.wbase : 0];
        for (int t = x.tid; t < nlw; t += nth) {
            const int row = t >> b.lgtx, col = t & (b.tilesx - 1);
            sp[t] = stage4(x.S.y + b.lsrc + row * x.G.ys32 + col * 4, b.satd_mode != 0);
        }
        if (b.chroma && b.cfast_src) {
            const int nc = b.ctilesx * b.crows;
            for (int t = x.tid; t < 2 * nc; t += nth) {
                const int pl = t >= nc, u = t - pl * nc;
                const int row = u >> b.lgctx, col = u & (b.ctilesx - 1);
                sp[nlw + t] = stage4((pl ? x.S.v : x.S.u) + b.csrc + row * x.G.cs32 + col * 4, x.satd != 0);
            }
        }
    }
}

// The refinement and bad-SAD expansion of one block (exact_refine_search :771-826,
// exact_hex2 :942-1033, exact_umh :1036-1119, the expansion :611-672): a state machine
// replicated in every thread of the direction, issuing one evaluation step at a time.
// (ppx, ppy): predictor of the motion penalty; (own_x, own_y): the block's own predictor,
// which the bad-SAD expansion switches to. `stage`: RS_ALL runs the refinement and the
// expansion, RS_REFINE_ONLY stops where the expansion's test begins, RS_BAD_ONLY starts
// there (the look-ahead runs the two apart: the test reads the bad count of the blocks
// committed before), RS_NONE runs nothing.
enum { RS_NONE, RS_ALL, RS_REFINE_ONLY, RS_BAD_ONLY };
template <class SH>
__device__ __forceinline__ void run_search_steps(const Ctx &x, const BlkC &b, SH &s, int &ph, int stage, int stype,
                                                 int radius, int lambda, int ppx, int ppy, int own_x, int own_y,
                                                 int64_t idx, int &bad_count, int &bmx, int &bmy, unsigned &bsad,
                                                 long long &bcost) {
    const AnalyseParams &P = *x.P;
    const LevelInfo &L = *x.L;
    const int level = x.level;
    int predx = ppx, predy = ppy;
    int state = stage == RS_NONE ? S_STORE : (stage == RS_BAD_ONLY ? S_BAD : S_REFINE);
    int hbx = 0, hby = 0, hdir = -2, hi = 0, hrad = 0, hret = 0, bad_r = 0, bad_max = 0;
    unsigned found = 0;
    for (;;) {
        Gen g{0, 0, 0, 0, 0, 0, 0};
        bool sets_mv = true, issue = false;
        while (!issue && state != S_STORE) {
            if (state == S_BAD && stage == RS_REFINE_ONLY) {
                state = S_STORE;
                break;
            }
            if (state == S_REFINE) {
                if (stype == 4) { g = make_gen(BK_EXH, bmx, bmy, radius, 0, 0); issue = true; state = S_BAD; }
                else if (stype == 3) {
                    g = make_gen(BK_UMH, bmx, bmy, radius, 0, 0); issue = true;
                    state = S_HEX_START; hrad = radius; hret = 0;
                } else if (stype == 2) { state = S_HEX_START; hrad = radius; hret = 0; }
                else state = S_BAD;
            } else if (state == S_HEX_START) {
                hbx = bmx; hby = bmy;
                if (hrad > 1) { g = make_gen(BK_HEX6, hbx, hby, 0, 0, 0); sets_mv = false; issue = true; state = S_HEX_ITER; }
                else { g = make_gen(BK_RING, hbx, hby, 1, 1, 0); issue = true; state = hret ? S_FINAL_RING : S_BAD; }
            } else if (state == S_HEX_ITER) {
                if (hi < hrad / 2 && hbx >= b.bnd0 && hby >= b.bnd1 && hbx < b.bnd2 && hby < b.bnd3) {
                    g = make_gen(BK_HEX3, hbx, hby, 0, 0, c_mod6m1[hdir + 1]); sets_mv = false; issue = true;
                } else state = S_HEX_EXIT;
            } else if (state == S_HEX_EXIT) {
                bmx = hbx; bmy = hby;
                g = make_gen(BK_RING, hbx, hby, 1, 1, 0); issue = true; state = hret ? S_FINAL_RING : S_BAD;
            } else if (state == S_BAD) {
                found = bsad;
                const int bl = sat_i32((long long)P.coarse_bad_sad + (long long)(sat_i32((long long)P.coarse_bad_sad * bad_count) / 16));
                if (level > 0 && idx > 1 && P.coarse_bad_sad > 0 && (int)bsad > bl) {
                    bad_count++;
                    predx = own_x; predy = own_y;  // the block's own predictor
                    if (P.coarse_bad_range < 0) {
                        bad_max = -P.coarse_bad_range * L.pel; bad_r = L.pel;
                        if (bad_r < bad_max) { g = make_gen(BK_RING, 0, 0, bad_r, L.pel, 0); issue = true; state = S_BAD_RING; }
                        else state = S_FINAL_RING;
                    } else if (P.coarse_bad_range > 0) {
                        hrad = P.coarse_bad_range * L.pel; hret = 1;
                        g = make_gen(BK_UMH, 0, 0, hrad, 0, 0); issue = true; state = S_HEX_START;
                    } else state = S_FINAL_RING;
                } else state = S_STORE;
            } else if (state == S_BAD_RING) {
                if (bsad < found / 4) state = S_FINAL_RING;
                else {
                    bad_r += L.pel;
                    if (bad_r < bad_max) { g = make_gen(BK_RING, 0, 0, bad_r, L.pel, 0); issue = true; }
                    else state = S_FINAL_RING;
                }
            } else {  // S_FINAL_RING
                g = make_gen(BK_RING, bmx, bmy, 1, 1, 0); issue = true; state = S_STORE;
            }
        }
        if (!issue) break;
        int w;
        eval_step(x, b, s, ph, g, lambda, predx, predy, bcost, bsad, w);
        if (g.kind == BK_HEX6 || g.kind == BK_HEX3) {  // exact_check_dir: a label, best.mv set at exit
            if (w >= 0) {
                hdir = g.kind == BK_HEX6 ? w : g.odir + w - 1;
                hbx += c_hex2[hdir + 1].x; hby += c_hex2[hdir + 1].y;
                hi = g.kind == BK_HEX6 ? 1 : hi + 1;
                state = S_HEX_ITER;
            } else state = S_HEX_EXIT;
        } else if (w >= 0 && sets_mv) {
            const int2 m = gen_mv(g, w);
            bmx = m.x; bmy = m.y;
        }
    }
}

// The per-direction search of one level (exact_search_level, :480-681). Every thread
// of the direction runs this with identical values; only the evaluation work is split.
__device__ __forceinline__ void search_level(const Ctx &x, DirSh &s, DirScratch &ds, const uint2 *prevp, int *status) {
    const AnalyseParams &P = *x.P;
    const LevelInfo &L = *x.L;
    const int level = x.level, gw = L.gw, gh = L.gh;
    const int64_t ncell = (int64_t)gw * gh;
    uint2 *field = ds.vec[level & 1];
    uint8_t *lumaf = ds.luma[level & 1];
    const int64_t order_len = s.order_len;
    const bool smallest = L.smallest != 0;
    const int lane = x.tid & 31, warp = x.tid >> 5;
    int bad_count = 0;
    int ph = 0;
    // The previous block's result: stored by thread 0 after the block's last barrier, so
    // the other warps take it from here until the next block's barrier publishes it.
    int64_t last_idx = -1;
    uint2 last_val = make_uint2(0, 0);
    for (int64_t k = 0; k < order_len; k++) {
        const int2 bxy = level == 0 ? initial_order_at(gw, gh, k) : unpack_xy(ds.order[k]);
        const int bx = bxy.x, by = bxy.y;
        const int64_t idx = (int64_t)by * gw + bx;
        int px = (level > 0 && bx == gw - 1) ? L.lw - P.block_w : bx * P.step_x;
        int py = (level > 0 && by == gh - 1) ? L.lh - P.block_h : by * P.step_y;
        px += L.pxoff;
        py += L.pyoff;
        const bool edge = level > 0 && (bx == gw - 1 || by == gh - 1);
        const int sxi = imin(bx, gw - 2), syi = imin(by, gh - 2);
        const int64_t sidx = (int64_t)syi * gw + sxi;
        if (sidx < 0 || sidx >= ncell || idx < 0 || idx >= ncell) {  // field[-1]: the reference panics
            if (x.tid == 0) { atomicOr(status, ST_PANIC); s.abort_ = 1; }
            break;
        }
        const int64_t fi = edge ? sidx : idx;
        const uint2 interp = fi == last_idx ? last_val : field[fi];
        const int2 imv = vmv(interp);
        BlkC b;
        make_blk(x, px, py, !smallest, b);
        stage_source(x, s, b);  // read by the refinement steps, after the next barrier
        // ---- special candidates (exact_search_block, :708-746): slot list in the
        // reference's evaluation roles; slot j is evaluated by group j
        int n = 0, rs_slot = -1, prev_slot = -1, nseeds = 0;
        int m0x = imv.x, m0y = imv.y;                    // slot 0: the interpolated predictor
        n = 1;
        if (edge && !smallest) rs_slot = n++;            // re-score the predictor at its source block (:536-549)
        int pmx = 0, pmy = 0;
        if (prevp) {
            const uint2 pv = prevp[idx];
            if (pv.y != 0xFFFFFFFFu && pv.y > 0) {
                const int2 pm = vmv(pv);
                pmx = pm.x; pmy = pm.y;
                prev_slot = n++;
            }
        }
        const int zslot = n++, gslot = n++, nslot0 = n;
        const int gxv = s.gx, gyv = s.gy;
        int sdx[8], sdy[8];
        bool panic = false;
        // the 3x3 neighbourhood: positions in the order and current vectors, loaded together
        int64_t npos[9];
        uint2 nval[9];
#pragma unroll
        for (int q = 0; q < 9; q++) {
            const int ny = by - 1 + q / 3, nx = bx - 1 + q % 3;
            npos[q] = 0x7FFFFFFFFFFFFFFFLL;
            nval[q] = make_uint2(0, 0);
            if (ny < 0 || ny >= gh || nx < 0 || nx >= gw) continue;
            const int64_t ci = (int64_t)ny * gw + nx;
            npos[q] = level == 0 ? initial_order_pos(gw, gh, nx, ny) : (int64_t)ds.pos[ci];
            nval[q] = ci == last_idx ? last_val : field[ci];
        }
#pragma unroll
        for (int q = 0; q < 9; q++) {
            const int64_t p = npos[q];
            if (p < k) {
                if (nseeds >= 8) { panic = true; continue; }  // seeds[8] overflows: the reference panics
                const int2 nm = vmv(nval[q]);
#pragma unroll
                for (int t = 0; t < 8; t++)
                    if (t == nseeds) { sdx[t] = nm.x; sdy[t] = nm.y; }
                nseeds++;
            }
        }
        if (panic) {
            if (x.tid == 0) { atomicOr(status, ST_PANIC); s.abort_ = 1; }
            break;
        }
        n += nseeds;
        const int dcslot = n++;
        // ---- evaluate the special slots
        const int G = step_lanes(x.grp_lanes, n, x.nw);
        const int grp = warp * (32 / G) + lane / G, sub = lane & (G - 1), NG = x.nw * (32 / G);
        unsigned (*slotL)[MAXSLOT] = s.slotL[x.wbase];
        for (int j0 = 0; j0 < n; j0 += NG) {
            const int j = j0 + grp;
            const bool act = j < n;
            int kind = 0, mx = 0, my = 0;
            bool ch = !smallest;
            if (j == 0) { mx = m0x; my = m0y; }
            else if (j == rs_slot) { mx = m0x; my = m0y; kind = 1; ch = true; }
            else if (j == prev_slot) { mx = pmx; my = pmy; }
            else if (j == zslot) { mx = 0; my = 0; }
            else if (j == gslot) { mx = gxv; my = gyv; }
            else if (j == dcslot) { kind = 2; ch = false; }
            else if (j >= nslot0 && j < nslot0 + nseeds) {
#pragma unroll
                for (int t = 0; t < 8; t++)
                    if (t == j - nslot0) { mx = sdx[t]; my = sdy[t]; }
            }
            Res r{0, 0, 0, 0, 0, 0};
            if (act) r = eval_lane(x, b, kind, sxi * P.step_x, syi * P.step_y, mx, my, ch, sub, G);
            group_sum3(r, G);
            if (act && sub == 0) {
                unsigned Lv, Cv;
                if (kind == 2) { Lv = r.L; Cv = 0; }
                else finalize(r, Lv, Cv);
                slotL[ph][j] = ch ? sat_add(Lv, Cv) : Lv;  // exact_sad: luma (+ chroma)
            }
        }
        gsync(x);
        const int phs = ph;
        ph ^= 1;
        // ---- selection among the special candidates (:716-747)
        const unsigned pred_score = rs_slot >= 0 ? slotL[phs][rs_slot] : interp.y;
        const bool field_valid = pred_score != 0xFFFFFFFFu;
        int bmx = 0, bmy = 0;
        unsigned bsad;
        long long bcost;
        bool refine = false;
        int lambda = 0, radius = 0, stype = 0, ppx = imv.x, ppy = imv.y;
        if (level == 0 && P.distance == 0) {
            if (field_valid) { bmx = imv.x; bmy = imv.y; bsad = slotL[phs][0]; }
            else bsad = slotL[phs][zslot];
            bcost = (long long)bsad;
        } else {
            if (field_valid) { bmx = imv.x; bmy = imv.y; bsad = slotL[phs][0]; bcost = (long long)bsad; }
            else { bsad = 0xFFFFFFFFu; bcost = 0x7FFFFFFFFFFFFFFFLL; }
            if (prev_slot >= 0) {
                const unsigned sd = slotL[phs][prev_slot];
                const long long cst = (long long)sd + (((long long)P.prev * sd) >> 8);
                if (cst < bcost) { bmx = pmx; bmy = pmy; bsad = sd; bcost = cst; ppx = pmx; ppy = pmy; }
            }
            {
                const unsigned sd = slotL[phs][gslot];
                const long long cst = (long long)sd + (((long long)P.pglobal * sd) >> 8);
                if (cst < bcost) { bmx = gxv; bmy = gyv; bsad = sd; bcost = cst; }
            }
            {
                const unsigned sd = slotL[phs][zslot];
                const long long cst = (long long)sd + (((long long)P.pzero * sd) >> 8);
                if (cst < bcost) { bmx = 0; bmy = 0; bsad = sd; bcost = cst; }
            }
#pragma unroll
            for (int q = 0; q < 8; q++) {
                if (q >= nseeds) break;
                const unsigned sd = slotL[phs][nslot0 + q];
                const long long cst = (long long)sd + (((long long)P.pnbour * sd) >> 8);
                if (cst < bcost) { bmx = sdx[q]; bmy = sdy[q]; bsad = sd; bcost = cst; }
            }
            bcost = (long long)bsad;
            lambda = adapt_lambda(L.lambda_base, L.lsad, pred_score);
            radius = L.base_radius;
            if (level > 0 && P.coarse_distance < 0) {
                const unsigned act = plane_activity(x.S.y, x.G.ylen, x.G.ys, L.y_off + b.py2, b.px2, b.bw, b.bh, x.satd) +
                                     plane_activity(x.S.u, x.G.clen, x.G.cs, L.c_off + py / 2, px / 2, b.bw / 2, b.bh / 2, x.satd) +
                                     plane_activity(x.S.v, x.G.clen, x.G.cs, L.c_off + py / 2, px / 2, b.bw / 2, b.bh / 2, x.satd);
                radius = adaptive_radius(radius, act);
            }
            stype = (edge && level == 1) ? 0 : L.search_type;
            refine = true;
        }
        const unsigned dcsum = slotL[phs][dcslot];
        run_search_steps(x, b, s, ph, refine ? RS_ALL : RS_NONE, stype, radius, lambda, ppx, ppy, imv.x, imv.y, idx,
                         bad_count, bmx, bmy, bsad, bcost);
        // ---- store (:673-679)
        const int rows = b.py >= 0 ? imax(0, imin(b.bh, L.lh - b.py)) : 0;
        const int cols = b.px >= 0 ? imax(0, imin(b.bw, L.lw - b.px)) : 0;
        const unsigned cnt = (unsigned)(rows * cols);
        unsigned dc = (cnt ? dcsum / cnt : 0) >> DC_SHIFT;
        if (dc > 255) dc = 255;
        const uint2 v = mkvec(bmx, bmy, smallest ? sat_mul(bsad, 3) : bsad);
        if (x.tid == 0) {
            field[idx] = v;
            lumaf[idx] = (uint8_t)dc;
        }
        last_idx = idx;
        last_val = v;
    }
}

// ---- level 0 with look-ahead (speculative and exact) ------------------------------------
// The calling warp waits until blocks 0 .. k-1 of the level are committed (*committed counts
// them; the committing warp stores its results, fences, then bumps the count). Bounded: false once
// kWaitCycles have passed or another warp of the direction has given up (the caller flags
// ST_TIMEOUT and carries on, so every warp still reaches its barriers). The fence after the wait
// makes the committed blocks' stores visible to every lane. XSM: the count and the stores it
// publishes are in global memory, written by warps on other SMs.
template <bool XSM>
__device__ __forceinline__ bool wait_commits(volatile int *committed, int64_t k, volatile int *late) {
    const long long t0 = clock64();
    for (;;) {
        const int seen = (int64_t)*committed >= k;
        if (__all_sync(0xFFFFFFFFu, seen)) break;
        const int give_up = *late || clock64() - t0 > kWaitCycles;
        if (__shfl_sync(0xFFFFFFFFu, give_up, 0)) {
            if ((threadIdx.x & 31) == 0) *late = 1;
            return false;
        }
        __nanosleep(32);
    }
    if (XSM) __threadfence();
    else __threadfence_block();
    return true;
}

// exact_search_level (:480-681) with D = NW blocks in flight per direction, one per warp
// ("look-ahead"). Warp w searches blocks w, w + D, w + 2D, ... of the level's order. Of what a
// block reads, only these can come from the blocks searched just before it: the vectors of its
// processed neighbours, taken as seeds (:570-585); at level > 0 an edge block's predictor, the
// current vector of an inner cell (:520-549); the bad-SAD count (:605-616). Everything else
// (the interpolated predictor of an inner block, lambda, radius, search type, the
// previous-frame, zero and global candidates) comes from the coarser level, the other direction
// and the block itself. A warp starts block k once it has committed block k - D, so cells
// processed at order positions <= k - D hold their final vectors; seeds from the at most D - 1
// cells processed at positions in (k - D, k) are "deferred": the block's special candidates and
// its refinement run without them. The warp then waits for block k - 1's commit (a count of
// committed blocks in shared memory: blocks commit in the reference's order) and replays the
// reference's selection
// with the deferred seeds at their places in the scan: :740-746 keep the first candidate of
// minimal cost, i.e. the least (cost, place), so the speculative best stands unless a deferred
// seed costs less, or the same at an earlier place. If one wins with another vector, the
// refinement runs again from it; with the same vector (hence the same SAD) the refinement
// already run is the reference's. The bad-SAD test and expansion run after the hand-over, with
// the count of the blocks before. An edge block whose predictor cell is among the deferred ones
// waits for block k - 1 first and runs without look-ahead. Stored vectors are the reference's in
// every case; on the 1080p workload fewer than 1 % of level-0 blocks run their refinement twice.
// A level with an input on which the reference would panic takes search_level instead.
// stats (nullable): [0] blocks, [1] blocks with deferred seeds, [2] deferred seeds evaluated
// (the others had the vector of a candidate already evaluated), [3] refinements run again.
//
// spec_walk is one warp's part: blocks g, g + D, ... of the level (x: a one-warp group; x.tid
// the lane). The count of committed blocks, the flag of a wait that gave up and the
// direction's abort flag are passed in: in shared memory when the direction's warps share a CTA
// (XSM false), in the pair's scratch when they are CTAs on different SMs (XSM true, the level-0
// kernel), where the field's cells written during the level are read from L2 (__ldcg: the SM's
// L1 is not coherent with the other SMs' stores) and commits fence device-wide.
template <bool XSM>
__device__ __forceinline__ uint2 ld_cell(const uint2 *p) {
    if (XSM) return __ldcg(p);
    return *p;
}
template <bool XSM, class SH>
__device__ __forceinline__ void spec_walk(const Ctx &x, SH &s, DirScratch &ds, const uint2 *prevp, int g, int64_t order_len,
                                          int gxv, int gyv, volatile int *committed, volatile int *late_flag,
                                          int *abort_flag, int *status, unsigned long long *stats) {
    const AnalyseParams &P = *x.P;
    const LevelInfo &L = *x.L;
    const int level = x.level, gw = L.gw, gh = L.gh;
    uint2 *field = ds.vec[level & 1];
    uint8_t *lumaf = ds.luma[level & 1];
    const bool smallest = L.smallest != 0;
    constexpr int D = NW;
    const int lane = x.tid;
    int ph = 0;
    unsigned long long n_blk = 0, n_def = 0, n_eval = 0, n_rerun = 0;
    bool late = false;
    unsigned (*slotL)[MAXSLOT] = s.slotL[x.wbase];
    auto wait_prev = [&](int64_t k) {  // block k - 1 is committed (and its stores visible) after this
        if (k > 0 && !wait_commits<XSM>(committed, k, late_flag)) late = true;
    };
    auto pos_of = [&](int nx, int ny) -> int64_t {
        return level == 0 ? initial_order_pos(gw, gh, nx, ny) : (int64_t)ds.pos[(int64_t)ny * gw + nx];
    };
    for (int64_t k = g; k < order_len; k += D) {
        const int2 bxy = level == 0 ? initial_order_at(gw, gh, k) : unpack_xy(ds.order[k]);
        const int bx = bxy.x, by = bxy.y;
        const int64_t idx = (int64_t)by * gw + bx;
        int px = (level > 0 && bx == gw - 1) ? L.lw - P.block_w : bx * P.step_x;
        int py = (level > 0 && by == gh - 1) ? L.lh - P.block_h : by * P.step_y;
        px += L.pxoff;
        py += L.pyoff;
        const bool edge = level > 0 && (bx == gw - 1 || by == gh - 1);
        const int sxi = imin(bx, gw - 2), syi = imin(by, gh - 2);
        const int64_t sidx = (int64_t)syi * gw + sxi;
        // an edge block's predictor is its inner cell's current vector: when another warp may not
        // have committed that cell yet, take the hand-over first (the block runs without look-ahead)
        bool waited = false;
        if (edge) {
            const int64_t p = pos_of(sxi, syi);
            if (p < k && p > k - D) { wait_prev(k); waited = true; }
        }
        const uint2 interp = ld_cell<XSM>(field + (edge ? sidx : idx));
        const int2 imv = vmv(interp);
        BlkC b;
        make_blk(x, px, py, !smallest, b);
        stage_source(x, s, b);
        // ---- special candidates (exact_search_block, :708-746), as in search_level, without
        // the deferred seeds
        int n = 1, rs_slot = -1, prev_slot = -1;
        if (edge && !smallest) rs_slot = n++;  // re-score the predictor at its source block (:536-549)
        int pmx = 0, pmy = 0;
        if (prevp) {
            const uint2 pv = prevp[idx];
            if (pv.y != 0xFFFFFFFFu && pv.y > 0) {
                const int2 pm = vmv(pv);
                pmx = pm.x; pmy = pm.y;
                prev_slot = n++;
            }
        }
        const int zslot = n++, gslot = n++, nslot0 = n;
        // seeds evaluated now and deferred seeds, in shared memory (written by lane 0; the values are
        // the same in every lane)
        int2 *sv = s.seedv[x.wbase];
        int *sq = s.seedq[x.wbase], *dq = s.defq[x.wbase];
        long long *dcell = s.defc[x.wbase];
        int nseeds = 0, nall = 0, ndef = 0;
#pragma unroll 1
        for (int q = 0; q < 9; q++) {
            const int ny = by - 1 + q / 3, nx = bx - 1 + q % 3;
            if (ny < 0 || ny >= gh || nx < 0 || nx >= gw) continue;
            const int64_t p = pos_of(nx, ny);
            if (p >= k) continue;
            const int64_t ci = (int64_t)ny * gw + nx;
            if (!waited && p > k - D) {  // searched by another warp, maybe not yet committed
                if (lane == 0) { dq[ndef] = nall; dcell[ndef] = ci; }
                ndef++;
            } else {
                const int2 nm = vmv(ld_cell<XSM>(field + ci));
                if (lane == 0) { sv[nseeds] = nm; sq[nseeds] = nall; }
                nseeds++;
            }
            nall++;  // at most 8: levels with more processed neighbours take search_level
        }
        __syncwarp();
        n += nseeds;
        const int dcslot = n++;
        {
            const int G = step_lanes(x.grp_lanes, n, 1);
            const int grp = lane / G, sub = lane & (G - 1), NG = 32 / G;
            for (int j0 = 0; j0 < n; j0 += NG) {
                const int j = j0 + grp;
                const bool act = j < n;
                int kind = 0, mx = 0, my = 0;
                bool ch = !smallest;
                if (j == 0) { mx = imv.x; my = imv.y; }
                else if (j == rs_slot) { mx = imv.x; my = imv.y; kind = 1; ch = true; }
                else if (j == prev_slot) { mx = pmx; my = pmy; }
                else if (j == zslot) { mx = 0; my = 0; }
                else if (j == gslot) { mx = gxv; my = gyv; }
                else if (j == dcslot) { kind = 2; ch = false; }
                else if (j >= nslot0 && j < nslot0 + nseeds) { mx = sv[j - nslot0].x; my = sv[j - nslot0].y; }
                Res r{0, 0, 0, 0, 0, 0};
                if (act) r = eval_lane(x, b, kind, sxi * P.step_x, syi * P.step_y, mx, my, ch, sub, G);
                group_sum3(r, G);
                if (act && sub == 0) {
                    unsigned Lv, Cv;
                    if (kind == 2) { Lv = r.L; Cv = 0; }
                    else finalize(r, Lv, Cv);
                    slotL[ph][j] = ch ? sat_add(Lv, Cv) : Lv;
                }
            }
        }
        __syncwarp();
        const int phs = ph;
        ph ^= 1;
        // ---- selection (:716-747); places in the reference's scan: field 0, previous 1,
        // global 2, zero 3, the neighbour seeds 4 + their place among the seeds
        const unsigned pred_score = rs_slot >= 0 ? slotL[phs][rs_slot] : interp.y;
        const bool field_valid = pred_score != 0xFFFFFFFFu;
        int bmx = 0, bmy = 0, bpos = -1;
        unsigned bsad;
        long long bcost;
        bool refine = false;
        int lambda = 0, radius = 0, stype = 0, ppx = imv.x, ppy = imv.y;
        if (level == 0 && P.distance == 0) {  // level 0 without a search: the field's vector or zero
            if (field_valid) { bmx = imv.x; bmy = imv.y; bsad = slotL[phs][0]; }
            else bsad = slotL[phs][zslot];
            bcost = (long long)bsad;
        } else {
            if (field_valid) { bmx = imv.x; bmy = imv.y; bsad = slotL[phs][0]; bcost = (long long)bsad; bpos = 0; }
            else { bsad = 0xFFFFFFFFu; bcost = 0x7FFFFFFFFFFFFFFFLL; }
            if (prev_slot >= 0) {
                const unsigned sd = slotL[phs][prev_slot];
                const long long cst = (long long)sd + (((long long)P.prev * sd) >> 8);
                if (cst < bcost) { bmx = pmx; bmy = pmy; bsad = sd; bcost = cst; ppx = pmx; ppy = pmy; bpos = 1; }
            }
            {
                const unsigned sd = slotL[phs][gslot];
                const long long cst = (long long)sd + (((long long)P.pglobal * sd) >> 8);
                if (cst < bcost) { bmx = gxv; bmy = gyv; bsad = sd; bcost = cst; bpos = 2; }
            }
            {
                const unsigned sd = slotL[phs][zslot];
                const long long cst = (long long)sd + (((long long)P.pzero * sd) >> 8);
                if (cst < bcost) { bmx = 0; bmy = 0; bsad = sd; bcost = cst; bpos = 3; }
            }
#pragma unroll 1
            for (int q = 0; q < nseeds; q++) {
                const unsigned sd = slotL[phs][nslot0 + q];
                const long long cst = (long long)sd + (((long long)P.pnbour * sd) >> 8);
                if (cst < bcost) { bmx = sv[q].x; bmy = sv[q].y; bsad = sd; bcost = cst; bpos = 4 + sq[q]; }
            }
            lambda = adapt_lambda(L.lambda_base, L.lsad, pred_score);
            radius = L.base_radius;
            if (level > 0 && P.coarse_distance < 0) {
                const unsigned act = plane_activity(x.S.y, x.G.ylen, x.G.ys, L.y_off + b.py2, b.px2, b.bw, b.bh, x.satd) +
                                     plane_activity(x.S.u, x.G.clen, x.G.cs, L.c_off + py / 2, px / 2, b.bw / 2, b.bh / 2, x.satd) +
                                     plane_activity(x.S.v, x.G.clen, x.G.cs, L.c_off + py / 2, px / 2, b.bw / 2, b.bh / 2, x.satd);
                radius = adaptive_radius(radius, act);
            }
            stype = (edge && level == 1) ? 0 : L.search_type;
            refine = true;
        }
        const long long sel_cost = bcost;
        const int sel_x = bmx, sel_y = bmy;
        bcost = (long long)bsad;
        const unsigned dcsum = slotL[phs][dcslot];
        // One call site of the search state machine (it is inlined, so each site is a copy of the
        // evaluation code): pass 0 the refinement with the seeds known at the start; pass 1 the
        // refinement again from a deferred seed that wins; pass 2 the bad-SAD test and expansion
        // (:604-672) with the count of the blocks committed before.
        int stage = refine ? RS_REFINE_ONLY : RS_NONE, pass = 0, bad_count = 0;
        for (;;) {
            run_search_steps(x, b, s, ph, stage, stype, radius, lambda, ppx, ppy, imv.x, imv.y, idx, bad_count, bmx,
                             bmy, bsad, bcost);
            if (pass == 0) {
                if (!waited) wait_prev(k);
                n_blk++;
                if (refine && ndef > 0) {
                    n_def++;
                    long long cb = sel_cost;
                    int cpos = bpos, cx = sel_x, cy = sel_y;
                    unsigned csad = 0;
                    bool dwin = false;
#pragma unroll 1
                    for (int j = 0; j < ndef; j++) {
                        const int64_t ci = dcell[j];
                        const int pos = 4 + dq[j];
                        const int2 m = vmv(ld_cell<XSM>(field + ci));
                        // its exact_sad: from an evaluated candidate with the same vector (same block,
                        // same reads), else evaluated now
                        unsigned sd = 0;
                        bool have = true;
                        if (m.x == imv.x && m.y == imv.y) sd = slotL[phs][0];
                        else if (prev_slot >= 0 && m.x == pmx && m.y == pmy) sd = slotL[phs][prev_slot];
                        else if (m.x == 0 && m.y == 0) sd = slotL[phs][zslot];
                        else if (m.x == gxv && m.y == gyv) sd = slotL[phs][gslot];
                        else {
                            have = false;
                            for (int t = 0; t < nseeds && !have; t++)
                                if (sv[t].x == m.x && sv[t].y == m.y) {
                                    sd = slotL[phs][nslot0 + t];
                                    have = true;
                                }
                        }
                        if (!have) {
                            Res r = eval_lane(x, b, 0, 0, 0, m.x, m.y, !smallest, lane, 32);
                            group_sum3(r, 32);
                            unsigned Lv, Cv;
                            finalize(r, Lv, Cv);
                            sd = !smallest ? sat_add(Lv, Cv) : Lv;
                            n_eval++;
                        }
                        const long long cst = (long long)sd + (((long long)P.pnbour * sd) >> 8);
                        if (cst < cb || (cst == cb && pos < cpos)) {
                            cb = cst; cpos = pos; cx = m.x; cy = m.y; csad = sd; dwin = true;
                        }
                    }
                    if (dwin && (cx != sel_x || cy != sel_y)) {  // a deferred seed with another vector wins
                        n_rerun++;
                        bmx = cx; bmy = cy; bsad = csad; bcost = (long long)csad;
                        pass = 1;
                        continue;
                    }
                }
            }
            if (pass < 2 && refine && level > 0) {
                bad_count = s.bad_count;
                stage = RS_BAD_ONLY;
                pass = 2;
                continue;
            }
            break;
        }
        if (pass == 2 && lane == 0) s.bad_count = bad_count;
        // ---- store (:673-679) and hand the order on to the next block's warp
        const int rows = b.py >= 0 ? imax(0, imin(b.bh, L.lh - b.py)) : 0;
        const int cols = b.px >= 0 ? imax(0, imin(b.bw, L.lw - b.px)) : 0;
        const unsigned cnt = (unsigned)(rows * cols);
        unsigned dc = (cnt ? dcsum / cnt : 0) >> DC_SHIFT;
        if (dc > 255) dc = 255;
        if (lane == 0) {
            field[idx] = mkvec(bmx, bmy, smallest ? sat_mul(bsad, 3) : bsad);
            lumaf[idx] = (uint8_t)dc;
            // the block's stores (and bad_count) before the count that publishes them
            if (XSM) __threadfence();
            else __threadfence_block();
            *committed = (int)(k + 1);
        }
        __syncwarp();
    }
    if (lane == 0) {
        if (late) { atomicOr(status, ST_TIMEOUT); *abort_flag = 1; }
        if (stats && level == 0) {
            atomicAdd(stats + 0, n_blk);
            atomicAdd(stats + 1, n_def);
            atomicAdd(stats + 2, n_eval);
            atomicAdd(stats + 3, n_rerun);
        }
    }
}
// The direction's warps of one CTA walk the level together (the count in shared memory).
__device__ __forceinline__ void search_level_spec(const Ctx &xd, DirSh &s, DirScratch &ds, const uint2 *prevp, int *status,
                                                  unsigned long long *stats) {
    if (xd.tid == 0) { s.committed = 0; s.late_ = 0; s.bad_count = 0; }
    dbar(xd.d);
    const int g = xd.tid >> 5;
    Ctx x = xd;
    x.nw = 1;
    x.wbase = g;
    x.tid = xd.tid & 31;
    spec_walk<false>(x, s, ds, prevp, g, s.order_len, s.gx, s.gy, &s.committed, &s.late_, &s.abort_, status, stats);
    dbar(xd.d);
}

// Whether search_level_spec may run this level: it takes neither the reference's panics
// (search_level reports them at the block where the reference stops) nor grids below 3 x 3.
// Called by every thread of the direction; the answer is the same in all of them.
__device__ __forceinline__ bool level_spec_ok(const Ctx &x, DirSh &s, DirScratch &ds) {
    const LevelInfo &L = *x.L;
    const int level = x.level, gw = L.gw, gh = L.gh;
    const int64_t ncell = (int64_t)gw * gh, order_len = s.order_len;
    if (gw < 3 || gh < 3) return false;
    if (x.tid == 0) s.unsafe_ = 0;
    dbar(x.d);
    int bad = 0;
    for (int64_t k = x.tid; k < order_len && !bad; k += NT) {
        const int2 bxy = level == 0 ? initial_order_at(gw, gh, k) : unpack_xy(ds.order[k]);
        const int bx = bxy.x, by = bxy.y;
        const int64_t idx = (int64_t)by * gw + bx;
        const int64_t sidx = (int64_t)imin(by, gh - 2) * gw + imin(bx, gw - 2);
        if (sidx < 0 || sidx >= ncell || idx < 0 || idx >= ncell || bx < 0 || by < 0 || bx >= gw || by >= gh) {
            bad = 1;
            break;
        }
        int nproc = 0;
        for (int q = 0; q < 9; q++) {
            const int ny = by - 1 + q / 3, nx = bx - 1 + q % 3;
            if (ny < 0 || ny >= gh || nx < 0 || nx >= gw) continue;
            const int64_t p = level == 0 ? initial_order_pos(gw, gh, nx, ny) : (int64_t)ds.pos[(int64_t)ny * gw + nx];
            nproc += p < k;
        }
        if (nproc > 8) bad = 1;
    }
    if (bad) s.unsafe_ = 1;
    dbar(x.d);
    const bool ok = s.unsafe_ == 0;
    dbar(x.d);
    return ok;
}

__device__ __forceinline__ long long floor_div(long long a, long long b) {  // i64::div_euclid for b > 0
    const long long q = a / b;
    return (a % b != 0 && a < 0) ? q - 1 : q;
}

// exact_recalculate (:1326-1451): when refine[0].thsad is set, the level-0 field is
// interpolated onto the half-size output blocks and each block whose interpolated score is
// above the threshold is searched again. Blocks do not read each other's results, so the
// visiting order does not matter; the direction's threads take them one after another with
// the same evaluation machinery as the hierarchy. Output: ds.vec[1] / ds.luma[1].
__device__ __forceinline__ void refine_pass(Ctx &x, DirSh &s, DirScratch &ds) {
    const AnalyseParams &P = *x.P;
    const uint2 *field = ds.vec[0];
    uint2 *out = ds.vec[1];
    uint8_t *outl = ds.luma[1];
    const int ogw = P.lv[0].gw, ogh = P.lv[0].gh;
    const int obw = P.block_w, obh = P.block_h, osx = P.step_x, osy = P.step_y;
    const int bw = P.out_bw, bh = P.out_bh;
    const int sx = imax(bw - P.out_ox, 1), sy = imax(bh - P.out_oy, 1);
    const int gw = P.out_gw, gh = P.out_gh;
    const int lw = P.lv[0].lw, lh = P.lv[0].lh;
    x.level = 0;
    x.pel = P.lv[0].pel;
    x.satd = P.refine_satd;
    int ph = 0;
    for (int by = 0; by < gh; by++) {
        for (int bx = 0; bx < gw; bx++) {
            const int cx = bw / 2 + sx * bx, cy = bh / 2 + sy * by;
            const int ox_ = (cx - obw / 2) / osx, oy_ = (cy - obh / 2) / osy;
            const long long dx_ = imax(cx - (obw / 2 + osx * ox_), 0), dy_ = imax(cy - (obh / 2 + osy * oy_), 0);
            const uint2 p00 = field[(int64_t)iclamp(oy_, 0, ogh - 1) * ogw + iclamp(ox_, 0, ogw - 1)];
            const uint2 p10 = field[(int64_t)iclamp(oy_, 0, ogh - 1) * ogw + iclamp(ox_ + 1, 0, ogw - 1)];
            const uint2 p01 = field[(int64_t)iclamp(oy_ + 1, 0, ogh - 1) * ogw + iclamp(ox_, 0, ogw - 1)];
            const uint2 p11 = field[(int64_t)iclamp(oy_ + 1, 0, ogh - 1) * ogw + iclamp(ox_ + 1, 0, ogw - 1)];
            auto interp = [&](long long a, long long b_, long long c, long long d) {
                const long long top = a * osx + dx_ * (b_ - a);
                const long long bottom = c * osx + dx_ * (d - c);
                return floor_div(top + floor_div(dy_ * (bottom - top), osy), osx);
            };
            const int2 m00 = vmv(p00), m10 = vmv(p10), m01 = vmv(p01), m11 = vmv(p11);
            const int mvx = (int)interp(m00.x, m10.x, m01.x, m11.x);
            const int mvy = (int)interp(m00.y, m10.y, m01.y, m11.y);
            const long long parent = interp(p00.y, p10.y, p01.y, p11.y) * (long long)(bw * bh) / (long long)(obw * obh);
            const int px = bx * sx, py = by * sy;
            const bool border = bx == 0 || by == 0 || bx == gw - 1 || by == gh - 1;
            const int factor = (border && bw > 4) ? 3 : 1;
            const int epx = px + (factor == 3 ? bw / 4 : 0), epy = py + (factor == 3 ? bh / 4 : 0);
            x.L = &P.rlv[factor == 3 ? 1 : 0];
            const LevelInfo &L = *x.L;
            x.tl = L.tl;
            x.tcp = L.tc;
            {
                const int T = L.tl + 2 * L.tc;
                const int tpl = iclamp(P.tiles_per_lane, 1, 8);
                const int want = (T + tpl - 1) / tpl;
                int g = 1;
                while (g < want && g < 32) g <<= 1;
                x.grp_lanes = g;
            }
            x.pnew = P.pnew / factor;
            BlkC b;
            make_blk(x, epx, epy, true, b);
            // exact_clip (:1269-1273) of the interpolated vector into mv_bounds
            const int pmx = iclamp(mvx, b.bnd0, imax(b.bnd2 - 1, b.bnd0)), pmy = iclamp(mvy, b.bnd1, imax(b.bnd3 - 1, b.bnd1));
            const int threshold = P.refine_thsad / factor;
            const bool search = parent > (long long)threshold;
            stage_source(x, s, b);
            {  // slot 0: exact_sad at the clipped predictor (when searching); slot 1: block_luma_dc
                const int Gl = step_lanes(x.grp_lanes, 2, x.nw), lane = x.tid & 31, grp = (x.tid >> 5) * (32 / Gl) + lane / Gl;
                const int sub = lane & (Gl - 1);
                const bool act = (grp == 0 && search) || grp == 1;
                Res r{0, 0, 0, 0, 0, 0};
                if (act) r = eval_lane(x, b, grp == 1 ? 2 : 0, 0, 0, pmx, pmy, grp == 0, sub, Gl);
                group_sum3(r, Gl);
                if (act && sub == 0) {
                    unsigned Lv, Cv;
                    if (grp == 1) { Lv = r.L; Cv = 0; }
                    else finalize(r, Lv, Cv);
                    s.slotL[x.wbase][ph][grp] = grp == 0 ? sat_add(Lv, Cv) : Lv;
                }
            }
            dbar(x.d);
            const int phs = ph;
            ph ^= 1;
            int bmx = pmx, bmy = pmy;
            unsigned bsad = parent < 0 ? 0u : (parent > 0xFFFFFFFFLL ? 0xFFFFFFFFu : (unsigned)parent);
            long long bcost = parent < 0 ? 0 : parent;
            if (search) {
                bsad = s.slotL[x.wbase][phs][0];
                bcost = (long long)bsad;
                const int lambda = by == 0 ? 0 : (P.lambda >> 2) / factor;
                int bad = 0;
                run_search_steps(x, b, s, ph, RS_ALL, P.refine_search_type, abs(P.refine_distance), lambda, pmx, pmy, pmx,
                                 pmy, 0, bad, bmx, bmy, bsad, bcost);
            }
            const unsigned dcsum = s.slotL[x.wbase][phs][1];
            const int rows = b.py >= 0 ? imax(0, imin(b.bh, lh - b.py)) : 0;
            const int cols = b.px >= 0 ? imax(0, imin(b.bw, lw - b.px)) : 0;
            const unsigned cnt = (unsigned)(rows * cols);
            unsigned dc = (cnt ? dcsum / cnt : 0) >> DC_SHIFT;
            if (dc > 255) dc = 255;
            if (x.tid == 0) {
                out[(int64_t)by * gw + bx] = mkvec(bmx, bmy, sat_mul(bsad, (unsigned)factor));
                outl[(int64_t)by * gw + bx] = (uint8_t)dc;
            }
        }
    }
    dbar(x.d);
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

// The hand-over words of one direction (AnalyseParams::off_ctl) when level 0 runs in the
// level-0 kernel: the pair kernel leaves the level with GO set (and the count, the global
// predictor and whether the other direction's projection exists); the level-0 kernel's warps
// count their commits in COMMITTED and flag a wait that gave up in LATE; ABORT, set by either,
// tells the finish kernel to leave the pair's payload unwritten (the status word says why).
enum { CTL_GO, CTL_COMMITTED, CTL_LATE, CTL_GX, CTL_GY, CTL_ABORT, CTL_PREV };

__device__ __forceinline__ DirScratch dir_scratch(const AnalyseParams &P, uint8_t *scr, int d) {
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
    return ds;
}

// The per-level fields of the search context. tpl_scale multiplies the 4x4 tiles a lane takes
// per candidate: the level-0 kernel's warps each search a block alone, where fewer, longer lane
// groups measured faster (two lanes per 16x16 SATD + chroma candidate: 209.4 -> 213.1 pairs/s;
// eight lanes: 186.4).
__device__ __forceinline__ void set_level(Ctx &x, const AnalyseParams &P, int level, int tpl_scale = 1) {
    const LevelInfo &L = P.lv[level];
    x.L = &L;
    x.level = level;
    x.satd = L.satd;
    x.pel = L.pel;
    x.G.lw = L.lw; x.G.lh = L.lh; x.G.clw = L.lw / 2; x.G.clh = L.lh / 2;
    x.G.ys = P.y_stride; x.G.cs = P.c_stride; x.G.ylen = P.y_len; x.G.clen = P.c_len;
    x.G.ys32 = (int)P.y_stride; x.G.cs32 = (int)P.c_stride;
    x.pnew = P.pnew;
    x.tl = L.tl;
    x.tcp = L.tc;
    {  // lanes per candidate: about `tiles_per_lane` 4x4 tiles per lane
        const int T = L.tl + (L.smallest ? 0 : 2 * L.tc);
        const int tpl = iclamp(P.tiles_per_lane, 1, 8) * tpl_scale;
        const int want = (T + tpl - 1) / tpl;
        int g = 1;
        while (g < want && g < 32) g <<= 1;
        x.grp_lanes = g;
    }
}

// Pair b of a launch (analyse_filter.rs:277-282: frame n pairs with min(n + delta, num_frames - 1)).
__device__ __forceinline__ PairRef pair_at(const PairSrc &psrc, int64_t pair) {
    if (psrc.table) return psrc.table[pair];
    const int64_t n = (int64_t)psrc.first + pair;
    int64_t n2 = n + psrc.delta;
    if (n2 > psrc.nframes - 1) n2 = psrc.nframes - 1;
    PairRef pr;
    pr.cur = psrc.clip + n * psrc.frame_bytes;
    pr.ref = psrc.clip + n2 * psrc.frame_bytes;
    return pr;
}

// One frame pair, both directions: the whole of analyse_pair (:68-226) plus the payload
// (:2740-2811). Called by every thread of the CTA; threads of a direction the
// configuration does not search (vectors 1 or 2 under a 2-direction batch CTA) only
// take part in the CTA-wide barriers. Status bits go to *status. split: a direction whose
// level 0 takes the look-ahead leaves it to the level-0 kernel (see CTL_GO) and the finish
// kernel packs the payload.
__device__ __forceinline__ void analyse_pair_dev(const AnalyseParams &P, const PairRef pr, uint8_t *__restrict__ pay,
                                                 uint8_t *__restrict__ scr, int *status, int &cta_abort,
                                                 unsigned long long *spec_stats, bool split) {
    extern __shared__ __align__(16) unsigned char smem[];
    const bool bidir = P.vectors == 3;
    const int half = (int)(threadIdx.x / NT);
    const bool idle = !bidir && half == 1;
    const int d = bidir ? half : ((P.vectors & 2) ? 0 : 1);  // 0 = forward (cur -> ref), 1 = backward
    const int tid = threadIdx.x % NT;
    DirSh &s = reinterpret_cast<DirSh *>(smem)[half];
    const px_t *src = (const px_t *)(d == 0 ? pr.cur : pr.ref);
    const px_t *ref = (const px_t *)(d == 0 ? pr.ref : pr.cur);
    DirScratch ds = dir_scratch(P, scr, d);
    int *ctl = (int *)(scr + P.off_ctl[d]);
    Ctx x;
    x.P = &P;
    x.d = half;
    x.tid = tid;
    x.nw = NW;
    x.wbase = 0;
    x.S = Planes{src, src + P.y_len, src + P.y_len + P.c_len};
    x.R = Planes{ref, ref + P.y_len, ref + P.y_len + P.c_len};
    if (threadIdx.x == 0) cta_abort = 0;
    if (tid == 0) { s.abort_ = idle ? 2 : 0; s.gx = 0; s.gy = 0; s.order_len = 0; }
    if (split && tid == 0 && !idle) { ctl[CTL_GO] = 0; ctl[CTL_ABORT] = 0; }
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
        // the coarser levels of a split launch: twice the tiles per lane (217.0 against 215.2 pairs/s)
        set_level(x, P, level, split && level > 0 ? 2 : 1);
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
            if (SVPF_LOOKAHEAD && NW > 1 && (P.lookahead & (level == 0 ? 1 : 2)) && level_spec_ok(x, s, ds)) {
                if (split && level == 0) {  // the level-0 kernel walks it
                    if (tid == 0) {
                        ctl[CTL_COMMITTED] = 0; ctl[CTL_LATE] = 0; ctl[CTL_GX] = s.gx; ctl[CTL_GY] = s.gy;
                        ctl[CTL_PREV] = prevp != nullptr; ctl[CTL_GO] = 1;
                    }
                } else {
                    search_level_spec(x, s, ds, prevp, status, spec_stats);
                }
            } else {
                search_level(x, s, ds, prevp, status);
            }
        }
        dbar(half);
        if (!s.abort_ && level > 0) {
            const uint2 *f = ds.vec[level & 1];
            global_doubled(x, s, f, ncell, ds.hist);
            reorder(x, s, f, gw, gh, ds, status);
        }
        pgw = gw; pgh = gh;
        if (tid == 0 && s.abort_ == 1) cta_abort = 1;
        __syncthreads();
    }
    if (split && tid == 0 && !idle && s.abort_ == 1) ctl[CTL_ABORT] = 1;
}

// After the hierarchy: the refine pass when configured, then rescale_scores (:2716-2738)
// and pack_vector_frame (:2740-2811). Out of line, called where little else is live, so
// neither adds to the hierarchy's register pressure. Every thread of the CTA calls it.
__device__ __noinline__ void finish_pair(const AnalyseParams *Pp, const PairRef pr, uint8_t *pay, uint8_t *scr) {
    extern __shared__ __align__(16) unsigned char smem[];
    const AnalyseParams &P = *Pp;
    const bool bidir = P.vectors == 3;
    const int half = (int)(threadIdx.x / NT);
    if (!bidir && half == 1) return;
    const int d = bidir ? half : ((P.vectors & 2) ? 0 : 1);
    const int tid = threadIdx.x % NT;
    DirSh &s = reinterpret_cast<DirSh *>(smem)[half];
    DirScratch ds = dir_scratch(P, scr, d);
    if (P.has_refine) {
        const px_t *src = (const px_t *)(d == 0 ? pr.cur : pr.ref);
        const px_t *ref = (const px_t *)(d == 0 ? pr.ref : pr.cur);
        Ctx x;
        x.P = &P;
        x.d = half;
        x.tid = tid;
        x.nw = NW;
        x.wbase = 0;
        x.S = Planes{src, src + P.y_len, src + P.y_len + P.c_len};
        x.R = Planes{ref, ref + P.y_len, ref + P.y_len + P.c_len};
        const LevelInfo &L0 = P.lv[0];
        x.G.lw = L0.lw; x.G.lh = L0.lh; x.G.clw = L0.lw / 2; x.G.clh = L0.lh / 2;
        x.G.ys = P.y_stride; x.G.cs = P.c_stride; x.G.ylen = P.y_len; x.G.clen = P.c_len;
        x.G.ys32 = (int)P.y_stride; x.G.cs32 = (int)P.c_stride;
        refine_pass(x, s, ds);
    }
    // ---- rescale_scores (:2716-2738) + pack_vector_frame (:2740-2811)
    const uint2 *f = ds.vec[P.has_refine ? 1 : 0];
    const uint8_t *fl = ds.luma[P.has_refine ? 1 : 0];
    const int64_t count = (int64_t)P.out_gw * P.out_gh;
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

// One CTA per frame pair. split: level 0 (where it takes the look-ahead) and the payload are
// left to analyse_level0_kernel and analyse_finish_kernel.
__global__ void __launch_bounds__(2 * NT, SVPF_MINB)
    analyse_kernel(const __grid_constant__ AnalyseParams P, const PairSrc psrc, uint8_t *__restrict__ payloads,
                   uint8_t *__restrict__ scratch, int *status, int split) {
    __shared__ int cta_abort;
    const int64_t pair = blockIdx.x;
    const PairRef pr = pair_at(psrc, pair);
    uint8_t *scr = scratch + pair * P.scratch_per_pair;
    analyse_pair_dev(P, pr, payloads + pair * P.payload_len, scr, status, cta_abort, psrc.stats, split != 0);
    __syncthreads();
    if (!split && !cta_abort) finish_pair(&P, pr, payloads + pair * P.payload_len, scr);
}

// Level 0 spread over the GPU: one CTA per warp of a search direction, (pair, direction, g) for
// the pairs first .. of the launch; warp g walks blocks g, g + NW, ... of the level exactly as
// the pair kernel's look-ahead does, but its partners run on other SMs, so every SM holds about
// the same number of walking warps whatever the pair count (one CTA per pair leaves some SMs
// with two pairs and others with one). The warps of a direction wait on one another, so the
// launch is cooperative: all its CTAs are resident at once, or it does not start.
constexpr int kLevel0Warps = 1;    // warps per CTA (of one direction)
constexpr int kLevel0TileScale = 2;  // see set_level
constexpr int kLevel0PerSM = 16;   // warps per SM: 128 registers per thread
__global__ void __launch_bounds__(32 * kLevel0Warps, kLevel0PerSM / kLevel0Warps)
    analyse_level0_kernel(const __grid_constant__ AnalyseParams P, const PairSrc psrc, int64_t first,
                          uint8_t *__restrict__ scratch, int *status) {
    __shared__ WarpSh sh[kLevel0Warps];
    constexpr int per_dir = NW / kLevel0Warps;  // CTAs per direction
    const int ndir = P.vectors == 3 ? 2 : 1;
    const int64_t pair = first + blockIdx.x / (ndir * per_dir);
    const int rem = (int)(blockIdx.x % (ndir * per_dir)), half = rem / per_dir;
    const int w = (int)(threadIdx.x >> 5), g = (rem % per_dir) * kLevel0Warps + w;
    WarpSh &s = sh[w];
    const int d = ndir == 2 ? half : ((P.vectors & 2) ? 0 : 1);
    uint8_t *scr = scratch + pair * P.scratch_per_pair;
    int *ctl = (int *)(scr + P.off_ctl[d]);
    if (!ctl[CTL_GO]) return;  // the pair kernel ran this level itself, or the direction stopped
    const PairRef pr = pair_at(psrc, pair);
    const px_t *src = (const px_t *)(d == 0 ? pr.cur : pr.ref);
    const px_t *ref = (const px_t *)(d == 0 ? pr.ref : pr.cur);
    DirScratch ds = dir_scratch(P, scr, d);
    Ctx x;
    x.P = &P;
    x.d = 0;
    x.tid = (int)(threadIdx.x & 31);
    x.nw = 1;
    x.wbase = 0;
    x.S = Planes{src, src + P.y_len, src + P.y_len + P.c_len};
    x.R = Planes{ref, ref + P.y_len, ref + P.y_len + P.c_len};
    set_level(x, P, 0, kLevel0TileScale);
    const int od = ndir == 2 ? 1 - d : d;
    const uint2 *prevp = ctl[CTL_PREV] ? (const uint2 *)(scr + P.off_proj[od][0]) : nullptr;
    spec_walk<true>(x, s, ds, prevp, g, initial_order_len(P.lv[0].gw, P.lv[0].gh), ctl[CTL_GX], ctl[CTL_GY],
                    ctl + CTL_COMMITTED, ctl + CTL_LATE, ctl + CTL_ABORT, status, psrc.stats);
}

// After the level-0 kernel: the refine pass, rescale and packing of every pair not stopped.
__global__ void __launch_bounds__(2 * NT, SVPF_MINB)
    analyse_finish_kernel(const __grid_constant__ AnalyseParams P, const PairSrc psrc, uint8_t *__restrict__ payloads,
                          uint8_t *__restrict__ scratch) {
    const int64_t pair = blockIdx.x;
    uint8_t *scr = scratch + pair * P.scratch_per_pair;
    const bool bidir = P.vectors == 3;
    const int d0 = bidir ? 0 : ((P.vectors & 2) ? 0 : 1);
    if (((const int *)(scr + P.off_ctl[d0]))[CTL_ABORT] || (bidir && ((const int *)(scr + P.off_ctl[1]))[CTL_ABORT]))
        return;
    finish_pair(&P, pair_at(psrc, pair), payloads + pair * P.payload_len, scr);
}

// Persistent form: a grid sized to the resident CTAs drains the item list in order (the
// host sorts it largest-first); each CTA pulls the next item with one atomic, copies the
// item's clip parameters into shared memory and runs the pair on its own scratch slot.
__global__ void __launch_bounds__(2 * NT, SVPF_MINB)
    analyse_batch_kernel(const AnalyseParams *__restrict__ clips, const BatchItem *__restrict__ items, int nitems,
                         unsigned *__restrict__ next_item, uint8_t *__restrict__ scratch, int64_t scratch_per_cta,
                         int *__restrict__ clip_status) {
    __shared__ int cta_abort;
    __shared__ int item_sh;
    __shared__ __align__(16) AnalyseParams P;
    uint8_t *scr = scratch + (int64_t)blockIdx.x * scratch_per_cta;
    for (;;) {
        if (threadIdx.x == 0) item_sh = (int)atomicAdd(next_item, 1u);
        __syncthreads();
        const int it = item_sh;
        if (it >= nitems) break;
        const BatchItem bi = items[it];
        {
            const int4 *src = reinterpret_cast<const int4 *>(clips + bi.clip);
            int4 *dst = reinterpret_cast<int4 *>(&P);
            for (int i = threadIdx.x; i < (int)(sizeof(AnalyseParams) / 16); i += blockDim.x) dst[i] = src[i];
        }
        __syncthreads();
        analyse_pair_dev(P, bi.pair, bi.payload, scr, clip_status + bi.clip, cta_abort, nullptr, false);
        __syncthreads();
        if (!cta_abort) finish_pair(&P, bi.pair, bi.payload, scr);
        __syncthreads();  // P, item_sh and the shared search state are reused by the next item
    }
}

}  // namespace

size_t dir_shared_bytes() { return sizeof(DirSh); }

cudaError_t prepare() {
    static cudaError_t once = [] {
        const int smem = (int)(2 * sizeof(DirSh));
        cudaError_t e = cudaFuncSetAttribute(analyse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(analyse_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(analyse_finish_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        return e;
    }();
    return once;
}

cudaError_t launch_plain(const AnalyseParams &P, const PairSrc &psrc, int npairs, uint8_t *payloads, uint8_t *scratch,
                         int *status_dev, cudaStream_t stream, int *launches) {
    if (npairs <= 0) return cudaSuccess;
    if (cudaError_t e = prepare()) return e;
    const int ndir = P.vectors == 3 ? 2 : 1;
    const bool split = SVPF_LOOKAHEAD && NW > 1 && (P.lookahead & 5) == 5;
    analyse_kernel<<<npairs, NT * ndir, sizeof(DirSh) * ndir, stream>>>(P, psrc, payloads, scratch, status_dev,
                                                                       split ? 1 : 0);
    if (launches) *launches += 1;
    if (!split) return cudaGetLastError();
    if (cudaError_t e = cudaGetLastError()) return e;
    // level 0: the CTAs of one launch wait on one another, so each launch takes the pairs whose
    // CTAs are all resident at once (one launch for up to 296 bidirectional pairs on 148 SMs)
    static const int resident = [] {
        int dev = 0, sms = 0, per_sm = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, analyse_level0_kernel, 32 * kLevel0Warps, 0) !=
                cudaSuccess)
            return 0;
        return sms * per_sm * kLevel0Warps;  // warps
    }();
    const int64_t most = resident / (ndir * NW);
    if (most < 1) return cudaErrorCooperativeLaunchTooLarge;
    const int64_t launches_needed = (npairs + most - 1) / most;
    const int64_t group = (npairs + launches_needed - 1) / launches_needed;  // even groups
    for (int64_t f = 0; f < npairs; f += group) {
        const int64_t n = npairs - f < group ? npairs - f : group;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)(n * ndir * NW / kLevel0Warps));
        cfg.blockDim = dim3(32 * kLevel0Warps);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        if (cudaError_t e = cudaLaunchKernelEx(&cfg, analyse_level0_kernel, P, psrc, f, scratch, status_dev)) return e;
        if (launches) *launches += 1;
    }
    analyse_finish_kernel<<<npairs, NT * ndir, sizeof(DirSh) * ndir, stream>>>(P, psrc, payloads, scratch);
    if (launches) *launches += 1;
    return cudaGetLastError();
}

cudaError_t batch_blocks_per_sm(int *blocks) {
    if (cudaError_t e = prepare()) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, analyse_batch_kernel, 2 * NT, 2 * sizeof(DirSh));
}

cudaError_t launch_batch(const AnalyseParams *clips_dev, const BatchItem *items_dev, int nitems, unsigned *next_item_dev,
                         uint8_t *scratch, int64_t scratch_per_cta, int *clip_status_dev, int grid, cudaStream_t stream,
                         int *launches) {
    if (nitems <= 0 || grid <= 0) return cudaSuccess;
    if (cudaError_t e = prepare()) return e;
    analyse_batch_kernel<<<grid, 2 * NT, 2 * sizeof(DirSh), stream>>>(clips_dev, items_dev, nitems, next_item_dev,
                                                                      scratch, scratch_per_cta, clip_status_dev);
    if (launches) *launches += 1;
    return cudaGetLastError();
}

}  // namespace SVPF_VARIANT
}  // namespace svpf
