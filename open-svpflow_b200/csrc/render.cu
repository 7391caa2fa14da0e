// render.cu -- SmoothFps's frame render on the device: the single warp of algorithms 1 and 2 and
// the two-source blends of algorithms 11, 13, 21, 22 and 23. Each output sample reads its source(s) at its
// position displaced by motion interpolated between the four motion-plane samples around it, and
// optionally blends with the undisplaced samples by the mode's mask.
//
// Follows crates/svpflow-core/src/renderer.rs: CpuRenderer::render_mode1_or_2 (:308-328) through
// render_selected_warp_rows (:876-984); render_mode11_or_13 and its zero-origin variant (:330-438)
// through render_dual_warp_rows (:1031-1172) and mode11_or_13_pixel (:2918-2943); render_mode21_or_22
// (:571-641) with mode21_pixel / mode22_pixel (:1830-1848); render_mode23 (:644-666) through
// render_mode23_plane_rows_inner (:1294-1537) with mode23_pixel (:1850-1868); set_threshold / set_threshold_value
// (:238-264), plane_params (:1539-1606), motion_samples (:1608-1638), render_tiles (:1925-2010),
// interpolate_row / interpolate_motion (:2582-2637), alpha_row / alpha_at_row / alpha_at_absolute
// (:2639-2722), interp_pair (:2724-2738), interpolation_weights / coeff (:2740-2770), plane_covers /
// plane_index (:2772-2790), tile_interior (:2809-2835), sample_plane (:2837-2861), max_mask
// (:2908-2915), mode1_pixel / mode13_pixel (:1818-1828), blend_255 / blend_256 / clamp_between
// (:3221-3231), cpu_map (:3186-3193). The reference walks tiles (one per vector block, plus a left
// column and a top row of width / height origin) and writes each tile's samples; here one thread
// owns kPx consecutive output samples of a row and finds their tile arithmetically: the last tile
// in the reference's loop order that covers them, since a later tile overwrites an earlier one where
// they overlap. The tile's motion is fetched once when the thread's samples share it; a thread runs
// kBatch batches of kPx samples and keeps the tile state between them.
//
// 32-bit arithmetic as the reference's scalar loops. Its x86-64 SSE tile paths keep 16-bit lanes,
// which give the same values for thresholds 0..256 (|motion| <= 1024, weights <= 32, mask values
// <= 255), the only thresholds accepted here.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "../../include/svpflow_b200.h"
#include "handles.h"

namespace {

constexpr int kLut = 2048, kMaxBlock = 32;
constexpr int kPx = 4;     // output samples per batch
constexpr int kBatch = 2;  // batches per thread: the tile state carries over when they share a tile

struct Source {  // a plain plane (shift 0) or a super clip's level 0 (sub-planes `span` bytes apart)
    const uint8_t *p;
    int64_t len, stride, span;
    int32_t covers;  // plane_covers
};

struct RenderPlane {
    Source src[2];
    uint8_t *dst;
    int64_t dst_stride;
    int32_t width, height, block_w, block_h, origin_x, origin_y, x_shift, y_shift, x_div, step;
    int32_t max_x, max_y;
    int32_t bw_log2, bh_log2;      // log2 of the block size when it is a power of two, else -1
    int32_t morigin_x, morigin_y;  // the plane's own origin (alpha_at_absolute's mask_params)
    int32_t xw[kMaxBlock][2], yw[kMaxBlock][2];
};

struct RenderJob {
    RenderPlane pl[3];
    const uint16_t *mx[4], *my[4];  // motion sets (set k reads source k & 1; the single warp uses set 0)
    const uint8_t *mask[3];         // the single warp: [0]; 11 / 13: [0], [1] of max_mask; 21 / 22: a, b, final
    int64_t mlen;
    int32_t grid_w, grid_h, interp, zero_origin, shift;
    int32_t lut_t[4];               // LUT factors of the sets: threshold or 256 - threshold
    int32_t threshold, mode13;      // the two-source blends
    int32_t mode22, threshold_limit;  // 21 / 22
};

// ---- host side: the renderer's per-plane constants
int32_t cpu_map(int32_t v) {
    static const int32_t m[32] = {0, 1, 2, 2, -1, 3, 3, 3, -1, -1, -1, 4, -1, 4, -1, 4,
                                  -1, -1, -1, -1, -1, -1, -1, -1, 5, -1, -1, -1, 5, -1, -1, 5};
    const int64_t i = (int64_t)v - 1;
    return (i >= 0 && i < 32) ? m[i] : -1;
}
int32_t sat32(int64_t v) { return v < INT32_MIN ? INT32_MIN : (v > INT32_MAX ? INT32_MAX : (int32_t)v); }
int32_t as_i32(double v) {  // Rust `as i32`
    if (v != v) return 0;
    if (v >= 2147483647.0) return INT32_MAX;
    if (v <= -2147483648.0) return INT32_MIN;
    return (int32_t)v;
}
void weights(int32_t total, int32_t shift, int32_t w[kMaxBlock][2]) {
    memset(w, 0, sizeof(int32_t) * 2 * kMaxBlock);
    if (total <= 0) return;
    const int32_t sh = shift < 0 ? 0 : shift;
    const int32_t scale = sh >= 32 ? 0 : (int32_t)(1u << sh);
    for (int32_t p = 0; p < total && p < kMaxBlock; p++) {
        if (shift < 0) { w[p][0] = total - p; w[p][1] = p; }
        else if (scale == 0) { w[p][0] = 1; w[p][1] = 0; }
        else {  // coeff: ceil(value * scale / total - 0.5) in f64, value * scale wrapping in 32 bits
            w[p][0] = as_i32(ceil((double)(int32_t)((uint32_t)(total - p) * (uint32_t)scale) / (double)total - 0.5));
            w[p][1] = as_i32(ceil((double)(int32_t)((uint32_t)p * (uint32_t)scale) / (double)total - 0.5));
        }
    }
}
int32_t sat_step_max(int32_t a, int32_t step) {  // a.saturating_mul(step).saturating_sub(1).max(0)
    const int32_t s = sat32((int64_t)sat32((int64_t)a * step) - 1);
    return s > 0 ? s : 0;
}
bool covers(const Source &s, int32_t shift, int32_t step, int32_t max_x, int32_t max_y) {  // plane_covers
    if (shift != 0 && (shift >= 31 || (1 << shift) != step)) return false;
    const uint64_t x = (uint64_t)max_x, y = (uint64_t)max_y;
    unsigned __int128 idx;
    if (shift == 0) {
        idx = (unsigned __int128)y * (uint64_t)s.stride + x;
    } else {
        const uint64_t mask = (1ull << shift) - 1;
        const uint64_t sub = ((y & mask) << shift) | (x & mask);
        idx = (unsigned __int128)sub * (uint64_t)s.span + (unsigned __int128)(y >> shift) * (uint64_t)s.stride +
              (x >> shift);
    }
    return idx < (unsigned __int128)(uint64_t)s.len;
}

// ---- device side
__device__ __forceinline__ int64_t src_index(const Source &s, int32_t shift, int32_t x, int32_t y) {
    if (shift == 0) return (int64_t)y * s.stride + x;
    const int32_t mask = (1 << shift) - 1;
    const int32_t sub = ((y & mask) << shift) | (x & mask);
    return (int64_t)sub * s.span + (int64_t)(y >> shift) * s.stride + (x >> shift);
}
__device__ __forceinline__ int32_t load(const Source &s, int64_t i) {
    return (i >= 0 && i < s.len) ? (int32_t)__ldg(s.p + i) : 0;
}
__device__ __forceinline__ int32_t interp_pair(int32_t a, int32_t b, int32_t total, int32_t shift, const int32_t *w) {
    const int32_t s = (int32_t)((uint32_t)w[0] * (uint32_t)a + (uint32_t)w[1] * (uint32_t)b);
    return shift < 0 ? s / total : s >> shift;
}
__device__ __forceinline__ int32_t clamp_byte(int32_t v) { return v < 0 ? 0 : (v > 255 ? 255 : v); }
__device__ __forceinline__ int32_t blend256(int32_t a, int32_t b, int32_t w) {
    return clamp_byte((a * (256 - w) + b * w) >> 8);
}
__device__ __forceinline__ int32_t blend255(int32_t a, int32_t b, int32_t w) {
    return clamp_byte((a * (255 - w) + b * w + 255) >> 8);
}
// The last tile of render_tiles' loop along one axis that covers `pos`: index g (-1 for the leading
// strip), its first sample and its length.
__device__ __forceinline__ void tile_of(int32_t pos, int32_t origin, int32_t blk, int32_t blk_log2, int32_t total,
                                        int32_t grid, int32_t &g, int32_t &base, int32_t &len) {
    g = pos < origin ? -1 : (blk_log2 >= 0 ? (pos - origin) >> blk_log2 : (pos - origin) / blk);
    if (g > grid - 1) g = grid - 1;
    base = g < 0 ? 0 : origin + blk * g;
    len = g < 0 ? origin : blk;
    if (base + blk >= total || g == grid - 1) len = total - base;
}
// motion_value: LUT entry k of set_threshold is trunc((k - 1024) * t / 256), computed here (no
// saturation for t in 0..256)
__device__ __forceinline__ int32_t motion(const RenderJob &J, const uint16_t *plane, int64_t i, int32_t t) {
    const int k = i < J.mlen ? __ldg(plane + i) : 1024;  // NEUTRAL beyond the plane
    return ((k < kLut - 1 ? k : kLut - 1) - 1024) * t / 256;
}
// a mask sample: sel < 0 -> the mode's mask, or max_mask of the two; sel >= 0 -> mask[sel]
__device__ __forceinline__ int32_t mask_at(const RenderJob &J, int sel, int64_t i) {
    if (i < 0 || i >= J.mlen) return 0;
    if (sel >= 0) return __ldg(J.mask[sel] + i);
    const int32_t a = __ldg(J.mask[0] + i);
    return J.mask[1] ? max(a, (int32_t)__ldg(J.mask[1] + i)) : a;
}
// alpha_at_absolute (renderer.rs:2687-2722): the mask's alpha on the zero-origin grid
__device__ __forceinline__ int32_t alpha_absolute(const RenderJob &J, const RenderPlane &p, int sel, int32_t x,
                                                  int32_t y) {
    const int32_t ox = p.morigin_x, oy = p.morigin_y, bw = p.block_w, bh = p.block_h;
    int32_t ix0 = 0, ix1 = 0, iy0 = 0, iy1 = 0;
    if (ox <= x) { ix0 = (x - ox) / bw; ix1 = ix0 + 1; }
    if (oy <= y) { iy0 = (y - oy) / bh; iy1 = iy0 + 1; }
    const int32_t fx = ox < x ? (x - ox) % bw : 0, fy = oy < y ? (y - oy) % bh : 0;
    const int64_t gw = J.grid_w;
    const int32_t tl = mask_at(J, sel, iy0 * gw + ix0), tr = mask_at(J, sel, iy0 * gw + ix1);
    const int32_t bl = mask_at(J, sel, iy1 * gw + ix0), br = mask_at(J, sel, iy1 * gw + ix1);
    const int32_t top = ((bw - fx) * tl + fx * tr) / bw, bottom = ((bw - fx) * bl + fx * br) / bw;
    return clamp_byte(((bh - fy) * top + fy * bottom) / bh);
}

struct Tile {  // one tile of render_tiles, seen from one output row
    int32_t bx, by, tw, th;
    int64_t i[4];  // motion-plane indices i00, i01, i10, i11
};
__device__ __forceinline__ Tile make_tile(const RenderJob &J, int32_t gx, int32_t bx, int32_t tw, int32_t gy,
                                          int32_t by, int32_t th) {
    Tile t;
    t.bx = bx; t.by = by; t.tw = tw; t.th = th;
    const int64_t gw = J.grid_w;
    t.i[0] = (int64_t)(gy > 0 ? gy : 0) * gw + (gx > 0 ? gx : 0);
    const int64_t nx = (gx >= 0 && gx != J.grid_w - 1) ? 1 : 0, ny = (gy >= 0 && gy != J.grid_h - 1) ? gw : 0;
    t.i[1] = t.i[0] + nx; t.i[2] = t.i[0] + ny; t.i[3] = t.i[0] + ny + nx;
    return t;
}

// One motion set over a tile (motion_samples), interpolated down to row py (interpolate_motion_row),
// with the extent of its four samples for tile_interior.
struct SetRow {
    int32_t rx0, rx1, ry0, ry1;
    int32_t mnx, mxx, mny, mxy;
};
__device__ __forceinline__ SetRow set_row(const RenderJob &J, const RenderPlane &p, const Tile &t, int set,
                                          int32_t py, const int32_t (*syw)[2]) {
    const bool c = p.x_div == 2;  // chroma: motion / 2 in both axes (4:2:0)
    const int32_t lt = J.lut_t[set];
    int32_t sx[4], sy[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int64_t i = J.interp ? t.i[q] : t.i[0];
        const int32_t mx = motion(J, J.mx[set], i, lt), my = motion(J, J.my[set], i, lt);
        sx[q] = c ? mx / 2 : mx;
        sy[q] = c ? my / 2 : my;
    }
    SetRow r;
    r.mnx = min(min(sx[0], sx[1]), min(sx[2], sx[3]));
    r.mxx = max(max(sx[0], sx[1]), max(sx[2], sx[3]));
    r.mny = min(min(sy[0], sy[1]), min(sy[2], sy[3]));
    r.mxy = max(max(sy[0], sy[1]), max(sy[2], sy[3]));
    if (J.interp) {
        const int32_t *wy = syw[min(py - t.by, kMaxBlock - 1)];
        r.rx0 = interp_pair(sx[0], sx[2], p.block_h, p.y_shift, wy);
        r.rx1 = interp_pair(sx[1], sx[3], p.block_h, p.y_shift, wy);
        r.ry0 = interp_pair(sy[0], sy[2], p.block_h, p.y_shift, wy);
        r.ry1 = interp_pair(sy[1], sy[3], p.block_h, p.y_shift, wy);
    } else {
        r.rx0 = r.rx1 = sx[0];
        r.ry0 = r.ry1 = sy[0];
    }
    return r;
}
// tile_interior for the sets read in a tile
__device__ __forceinline__ bool interior(const RenderPlane &p, const Tile &t, const SetRow &r) {
    const int64_t st = p.step;
    return (int64_t)t.bx * st + r.mnx >= 0 && (int64_t)t.by * st + r.mny >= 0 &&
           (int64_t)(t.bx + t.tw - 1) * st + r.mxx <= p.max_x && (int64_t)(t.by + t.th - 1) * st + r.mxy <= p.max_y;
}
// the mask interpolated down to row py (alpha_row)
__device__ __forceinline__ void mask_row(const RenderJob &J, const RenderPlane &p, const Tile &t, int32_t py,
                                         const int32_t (*syw)[2], int sel, int32_t &m0, int32_t &m1) {
    const int32_t a = mask_at(J, sel, t.i[0]), b = mask_at(J, sel, t.i[1]), cc = mask_at(J, sel, t.i[2]),
                  d = mask_at(J, sel, t.i[3]);
    if (J.interp) {
        const int32_t *wy = syw[min(py - t.by, kMaxBlock - 1)];
        m0 = interp_pair(a, cc, p.block_h, p.y_shift, wy);
        m1 = interp_pair(b, d, p.block_h, p.y_shift, wy);
    } else {
        m0 = m1 = a;
    }
}
// a sample's displaced source position (interpolate_motion, then sample_plane's direct or clamped read)
__device__ __forceinline__ int64_t warp_index(const RenderJob &J, const RenderPlane &p, const Source &s,
                                              const SetRow &r, bool direct, int32_t px, int32_t bx, int32_t py,
                                              const int32_t (*sxw)[2]) {
    int32_t dx = r.rx0, dy = r.ry0;
    if (J.interp) {
        const int32_t *wx = sxw[min(px - bx, kMaxBlock - 1)];
        dx = interp_pair(r.rx0, r.rx1, p.block_w, p.x_shift, wx);
        dy = interp_pair(r.ry0, r.ry1, p.block_w, p.x_shift, wx);
    }
    int32_t xs = px * p.step + dx, ys = py * p.step + dy;
    if (!direct) {
        xs = min(max(xs, 0), p.max_x);
        ys = min(max(ys, 0), p.max_y);
    }
    return src_index(s, J.shift, xs, ys);
}
// the mask's alpha at a sample (alpha_at_absolute on the zero-origin grid, else alpha_at_row)
__device__ __forceinline__ int32_t alpha_at(const RenderJob &J, const RenderPlane &p, int sel, int32_t m0,
                                            int32_t m1, int32_t px, int32_t bx, int32_t py, const int32_t (*sxw)[2]) {
    if (J.zero_origin) return alpha_absolute(J, p, sel, px, py);
    if (!J.interp) return clamp_byte(m0);
    return clamp_byte(interp_pair(m0, m1, p.block_w, p.x_shift, sxw[min(px - bx, kMaxBlock - 1)]));
}

// KIND 0: the single warp (source 0, set 0; mode1_pixel with the mask when MASK). KIND 1: the
// two-source blend of algorithms 11 / 13 (set 0 reads source 0, set 1 source 1; mode11_or_13_pixel,
// max_mask when MASK). KIND 2: algorithms 21 / 22 (the same reads; mode21_or_22_pixel with alphas from
// masks a and b, and the final mask when MASK). KIND 3: algorithm 23 (sets base0, base1, next0, prev1,
// set k reading source k & 1; mode23_pixel with masks a and b, and the final mask when MASK).
// Grid: (row length of the widest plane / (256 kPx kBatch), rows of the tallest plane, 3 planes).
// Resident CTAs per SM the registers are budgeted for, per kind, as measured on 1080p frames: the
// masked two-source kinds gain a third CTA at 80 registers (algorithm 21: +31 %; a fourth at 64
// spills and loses 4 %); algorithm 23 spills at 80 and keeps two.
template <int KIND, bool MASK>
__global__ void __launch_bounds__(256, KIND == 0 ? (MASK ? 4 : 5) : (KIND == 1 ? (MASK ? 3 : 4) : (KIND == 2 ? 3 : 2)))
    render_kernel(const __grid_constant__ RenderJob J) {
    constexpr bool DUAL = KIND > 0;
    constexpr int NS = KIND == 0 ? 1 : (KIND == 3 ? 4 : 2);          // motion sets
    constexpr int NA = KIND >= 2 ? (MASK ? 3 : 2) : (MASK ? 1 : 0);  // alphas per sample
    const RenderPlane &p = J.pl[blockIdx.z];
    // the plane's interpolation weights in shared memory (indexed per thread)
    __shared__ int32_t sxw[kMaxBlock][2], syw[kMaxBlock][2];
    for (int t = threadIdx.x; t < 4 * kMaxBlock; t += blockDim.x) {
        if (t < 2 * kMaxBlock) (&sxw[0][0])[t] = (&p.xw[0][0])[t];
        else (&syw[0][0])[t - 2 * kMaxBlock] = (&p.yw[0][0])[t - 2 * kMaxBlock];
    }
    __syncthreads();
    const int32_t py = blockIdx.y;
    const int32_t pxa = (blockIdx.x * blockDim.x + threadIdx.x) * (kPx * kBatch);
    if (pxa >= p.width || py >= p.height || p.block_w <= 0 || p.block_h <= 0) return;
    int32_t gy, by, th;
    tile_of(py, p.origin_y, p.block_h, p.bh_log2, p.height, J.grid_h, gy, by, th);
    int32_t gx, bx, tw;
    tile_of(pxa, p.origin_x, p.block_w, p.bw_log2, p.width, J.grid_w, gx, bx, tw);
    Tile t = make_tile(J, gx, bx, tw, gy, by, th);
    SetRow r[NS];
#pragma unroll
    for (int k = 0; k < NS; k++) r[k] = set_row(J, p, t, k, py, syw);
    // the mask selectors of the alphas: the mode's (max) mask, or masks a, b, final
    auto sel_of = [](int a) { return KIND >= 2 ? a : -1; };
    int32_t m0[NA > 0 ? NA : 1], m1[NA > 0 ? NA : 1];
#pragma unroll
    for (int a = 0; a < NA; a++) mask_row(J, p, t, py, syw, sel_of(a), m0[a], m1[a]);
    auto direct_of = [&]() {  // plane_covers && tile_interior for the tile's sets
        bool d = p.src[0].covers && p.step > 0 && (!DUAL || p.src[1].covers);
#pragma unroll
        for (int k = 0; k < NS; k++) d = d && interior(p, t, r[k]);
        return d;
    };
    bool direct = direct_of();
    for (int bt = 0; bt < kBatch; bt++) {
    const int32_t px0 = pxa + bt * kPx;
    if (px0 >= p.width) break;
    const int32_t pxl = min(px0 + kPx - 1, p.width - 1);
    int32_t gxl, bxl, twl;
    if (bt > 0) {  // the batch's first sample may start another tile
        tile_of(px0, p.origin_x, p.block_w, p.bw_log2, p.width, J.grid_w, gxl, bxl, twl);
        if (gxl != gx) {
            gx = gxl;
            t = make_tile(J, gxl, bxl, twl, gy, by, th);
#pragma unroll
            for (int q = 0; q < NS; q++) r[q] = set_row(J, p, t, q, py, syw);
#pragma unroll
            for (int a = 0; a < NA; a++) mask_row(J, p, t, py, syw, sel_of(a), m0[a], m1[a]);
            direct = direct_of();
        }
    }
    tile_of(pxl, p.origin_x, p.block_w, p.bw_log2, p.width, J.grid_w, gxl, bxl, twl);
    const bool shared_tile = gx == gxl;  // usually: then the tile's motion is fetched once
    // indices first, then every load of the batch's samples, so the gathers overlap
    int64_t idx[NS][kPx];
    int32_t alpha[NA > 0 ? NA : 1][kPx];
#pragma unroll
    for (int k = 0; k < kPx; k++) {
        const int32_t px = px0 + k;
#pragma unroll
        for (int q = 0; q < NS; q++) idx[q][k] = -1;
#pragma unroll
        for (int a = 0; a < NA; a++) alpha[a][k] = 0;
        if (px > pxl) continue;
        if (!shared_tile && k > 0) {
            int32_t gk, bk, twk;
            tile_of(px, p.origin_x, p.block_w, p.bw_log2, p.width, J.grid_w, gk, bk, twk);
            if (gk != gx) {
                gx = gk;
                t = make_tile(J, gk, bk, twk, gy, by, th);
#pragma unroll
                for (int q = 0; q < NS; q++) r[q] = set_row(J, p, t, q, py, syw);
#pragma unroll
                for (int a = 0; a < NA; a++) mask_row(J, p, t, py, syw, sel_of(a), m0[a], m1[a]);
                direct = direct_of();
            }
        }
#pragma unroll
        for (int q = 0; q < NS; q++) idx[q][k] = warp_index(J, p, p.src[q & 1], r[q], direct, px, t.bx, py, sxw);
#pragma unroll
        for (int a = 0; a < NA; a++) alpha[a][k] = alpha_at(J, p, sel_of(a), m0[a], m1[a], px, t.bx, py, sxw);
    }
    // the undisplaced samples (px * step <= max_x: no clamp)
    const bool bases = KIND == 0 ? MASK : (KIND == 1 ? (MASK || J.mode13) : (KIND == 2 ? (MASK || J.mode22) : MASK));
    int32_t v[NS][kPx], c0[kPx], c1[kPx];
#pragma unroll
    for (int k = 0; k < kPx; k++) {
        const int32_t px = min(px0 + k, pxl);
#pragma unroll
        for (int q = 0; q < NS; q++) v[q][k] = load(p.src[q & 1], idx[q][k]);
        c0[k] = bases ? load(p.src[0], src_index(p.src[0], J.shift, px * p.step, py * p.step)) : 0;
        c1[k] = bases && DUAL ? load(p.src[1], src_index(p.src[1], J.shift, px * p.step, py * p.step)) : 0;
    }
    int32_t out[kPx];
#pragma unroll
    for (int k = 0; k < kPx; k++) {
        int32_t o;
        if (KIND == 3) {  // mode23_pixel: a, b, c, d = base0, base1, next0, prev1 samples
            const int32_t a = v[0][k], b = v[1 % NS][k], c = v[2 % NS][k], d = v[3 % NS][k];
            const int32_t lo = min(a, b), hi = max(a, b);
            const int32_t i0 = blend255(a, min(max(d, lo), hi), alpha[0][k]);
            const int32_t i1 = blend255(b, min(max(c, lo), hi), alpha[1 % NA][k]);
            o = blend256(i0, i1, J.threshold);
            if (MASK) o = blend255(o, blend256(c0[k], c1[k], J.threshold), alpha[NA - 1][k]);
        } else if (KIND == 2) {  // mode21_or_22_pixel
            const int32_t v0 = v[0][k], v1 = v[1 % NS][k];
            const int32_t ea = blend255(v0, v1, alpha[0][k]), eb = blend255(v1, v0, alpha[1 % NA][k]);
            if (J.mode22) o = min(max(blend256(c0[k], c1[k], J.threshold), min(ea, eb)), max(ea, eb));
            else o = blend256(ea, eb, J.threshold);
            if (MASK) o = blend255(o, blend256(c0[k], c1[k], J.threshold_limit), alpha[NA - 1][k]);
        } else if (KIND == 1) {  // mode11_or_13_pixel
            const int32_t v0 = v[0][k], v1 = v[1 % NS][k];
            const int32_t bl = blend256(c0[k], c1[k], J.threshold);
            if (J.mode13) o = min(max(bl, min(v0, v1)), max(v0, v1));  // mode13_pixel
            else o = blend256(v0, v1, J.threshold);                     // mode11_pixel
            if (MASK) o = blend255(o, bl, alpha[0][k]);
        } else {
            o = MASK ? blend255(v[0][k], c0[k], alpha[0][k]) : v[0][k];  // mode1_pixel
        }
        out[k] = o;
    }
    uint8_t *dst = p.dst + (int64_t)py * p.dst_stride + px0;
#pragma unroll
    for (int k = 0; k < kPx; k++)
        if (px0 + k <= pxl) dst[k] = (uint8_t)out[k];
    }
}

// Per-plane constants of one frame (plane_params for chroma = plane > 0), the sources' layouts and
// plane_covers; validation of the caller's arguments.
int setup(RenderJob &J, const svpf_render_config *cfg, int nsrc, const uint8_t *const *const src[2],
          const int64_t *const stride[2], const int64_t *const len[2], int32_t src_shift, uint8_t *const dst[3],
          const int64_t dst_stride[3], int32_t &most_w, int32_t &most_h) {
    const int32_t cd = 2;  // SmoothFps renders 4:2:0 (CpuConfig::chroma_y_div)
    J.mlen = (int64_t)cfg->grid_w * cfg->grid_h;
    J.grid_w = cfg->grid_w;
    J.grid_h = cfg->grid_h;
    J.shift = src_shift;
    most_w = most_h = 0;
    for (int pl = 0; pl < 3; pl++) {
        RenderPlane &p = J.pl[pl];
        const bool c = pl > 0;
        p.dst = dst[pl];
        p.dst_stride = dst_stride[pl];
        p.width = c ? cfg->width / 2 : cfg->width;
        p.height = c ? cfg->height / cd : cfg->height;
        p.block_w = c ? cfg->block_w / 2 : cfg->block_w;
        p.block_h = c ? cfg->block_h / cd : cfg->block_h;
        p.morigin_x = c ? cfg->origin_x / 2 : cfg->origin_x;
        p.morigin_y = c ? cfg->origin_y / cd : cfg->origin_y;
        p.origin_x = J.zero_origin ? 0 : p.morigin_x;
        p.origin_y = J.zero_origin ? 0 : p.morigin_y;
        p.x_shift = cpu_map(c ? cfg->block_w / 2 : cfg->block_w);
        p.y_shift = cpu_map(c ? cfg->block_h / 2 : cfg->block_h);
        p.x_div = c ? 2 : 1;
        p.step = cfg->source_step;
        p.max_x = sat_step_max(p.width, p.step);
        p.max_y = sat_step_max(p.height, p.step);
        weights(p.block_w, p.x_shift, p.xw);
        weights(p.block_h, p.y_shift, p.yw);
        p.bw_log2 = p.block_w > 0 && (p.block_w & (p.block_w - 1)) == 0 ? 31 - __builtin_clz((unsigned)p.block_w) : -1;
        p.bh_log2 = p.block_h > 0 && (p.block_h & (p.block_h - 1)) == 0 ? 31 - __builtin_clz((unsigned)p.block_h) : -1;
        if (!p.dst || p.dst_stride < p.width) return SVPF_EINVAL;
        for (int s = 0; s < nsrc; s++) {
            Source &S = p.src[s];
            S.p = src[s][pl];
            S.len = len[s][pl];
            S.stride = stride[s][pl];
            S.span = S.stride * p.height;  // sub-planes of a super clip's level 0
            if (!S.p || S.stride < 0 || S.len < 0) return SVPF_EINVAL;
            S.covers = covers(S, src_shift, p.step, p.max_x, p.max_y);
        }
        if (p.block_w > 0 && p.block_h > 0) {
            most_w = p.width > most_w ? p.width : most_w;
            most_h = p.height > most_h ? p.height : most_h;
        }
    }
    return SVPF_OK;
}

int check_common(const svpf_render_config *cfg, int32_t threshold, int32_t src_shift) {
    if (int rc = svpf::require_device()) return rc;
    if (!cfg) {
        svpf::set_last_error("render: null argument");
        return SVPF_EINVAL;
    }
    if (threshold < 0 || threshold > 256) {
        svpf::set_last_error("render: threshold must be 0..256");
        return SVPF_EINVAL;
    }
    if (src_shift < 0 || src_shift > 2 || (src_shift > 0 && (1 << src_shift) != cfg->source_step)) {
        svpf::set_last_error("render: super-plane shift must be log2(source_step), pel 1, 2 or 4");
        return SVPF_EINVAL;
    }
    return SVPF_OK;
}
bool draws_nothing(const svpf_render_config *cfg) {  // render_tiles returns at once
    return cfg->width <= 0 || cfg->height <= 0 || cfg->grid_w <= 0 || cfg->grid_h <= 0 || cfg->source_step <= 0 ||
           cfg->block_w <= 0 || cfg->block_h <= 0;
}
int launch(const RenderJob &J, int kind, bool mask, int32_t most_w, int32_t most_h, void *stream) {
    for (int k = 0; k < 4; k++)  // uint16 loads from an odd address would fault
        if (((uintptr_t)J.mx[k] | (uintptr_t)J.my[k]) & 1) {
            svpf::set_last_error("render: motion planes must be 2-byte aligned");
            return SVPF_EINVAL;
        }
    cudaError_t e = cudaSuccess;
    if (most_w > 0 && most_h > 0) {
        dim3 grid((unsigned)((most_w + 256 * kPx * kBatch - 1) / (256 * kPx * kBatch)), (unsigned)most_h, 3);
        cudaStream_t st = (cudaStream_t)stream;
        if (kind == 3) {
            if (mask) render_kernel<3, true><<<grid, 256, 0, st>>>(J);
            else render_kernel<3, false><<<grid, 256, 0, st>>>(J);
        } else if (kind == 2) {
            if (mask) render_kernel<2, true><<<grid, 256, 0, st>>>(J);
            else render_kernel<2, false><<<grid, 256, 0, st>>>(J);
        } else if (kind == 1) {
            if (mask) render_kernel<1, true><<<grid, 256, 0, st>>>(J);
            else render_kernel<1, false><<<grid, 256, 0, st>>>(J);
        } else {
            if (mask) render_kernel<0, true><<<grid, 256, 0, st>>>(J);
            else render_kernel<0, false><<<grid, 256, 0, st>>>(J);
        }
        svpf::add_launches(1);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        svpf::set_last_error(std::string("render: ") + cudaGetErrorString(e));
        return SVPF_ECUDA;
    }
    return SVPF_OK;
}

}  // namespace

extern "C" {

int svpf_render_warp_device(const svpf_render_config *cfg, int32_t threshold, int32_t mode1, int32_t interp,
                            const uint8_t *const src[3], const int64_t src_stride[3], const int64_t src_len[3],
                            int32_t src_shift, const uint16_t *motion_x, const uint16_t *motion_y,
                            const uint8_t *mask, uint8_t *const dst[3], const int64_t dst_stride[3], void *stream) {
    if (int rc = check_common(cfg, threshold, src_shift)) return rc;
    if (!src || !src_stride || !src_len || !dst || !dst_stride || !motion_x || !motion_y) {
        svpf::set_last_error("render: null argument");
        return SVPF_EINVAL;
    }
    if (draws_nothing(cfg)) return SVPF_OK;
    RenderJob *J = new RenderJob;
    memset(J, 0, sizeof(*J));
    // set_threshold: mode 1 warps with the inverse LUT, mode 2 with the threshold LUT
    J->lut_t[0] = mode1 ? 256 - threshold : threshold;
    J->mx[0] = motion_x;
    J->my[0] = motion_y;
    J->mask[0] = mask;
    J->interp = interp != 0;
    J->zero_origin = interp == 0;  // plane_params(chroma, zero_origin = !interp)
    const uint8_t *const *srcs[2] = {src, nullptr};
    const int64_t *strides[2] = {src_stride, nullptr}, *lens[2] = {src_len, nullptr};
    int32_t mw, mh;
    int rc = setup(*J, cfg, 1, srcs, strides, lens, src_shift, dst, dst_stride, mw, mh);
    if (rc) svpf::set_last_error("render: bad plane buffers");
    else rc = launch(*J, 0, mask != nullptr, mw, mh, stream);
    delete J;
    return rc;
}

int svpf_render_blend_device(const svpf_render_config *cfg, int32_t threshold, int32_t mode13, int32_t interp,
                             int32_t zero_origin, const uint8_t *const src0[3], const int64_t src0_stride[3],
                             const int64_t src0_len[3], const uint8_t *const src1[3], const int64_t src1_stride[3],
                             const int64_t src1_len[3], int32_t src_shift, const uint16_t *motion0_x,
                             const uint16_t *motion0_y, const uint16_t *motion1_x, const uint16_t *motion1_y,
                             const uint8_t *mask_a, const uint8_t *mask_b, uint8_t *const dst[3],
                             const int64_t dst_stride[3], void *stream) {
    if (int rc = check_common(cfg, threshold, src_shift)) return rc;
    if (!src0 || !src0_stride || !src0_len || !src1 || !src1_stride || !src1_len || !dst || !dst_stride ||
        !motion0_x || !motion0_y || !motion1_x || !motion1_y || (!mask_a) != (!mask_b)) {
        svpf::set_last_error("render: null argument (masks: both or neither)");
        return SVPF_EINVAL;
    }
    if (draws_nothing(cfg)) return SVPF_OK;
    RenderJob *J = new RenderJob;
    memset(J, 0, sizeof(*J));
    J->lut_t[0] = threshold;        // motion0 with the threshold LUT
    J->lut_t[1] = 256 - threshold;  // motion1 with the inverse LUT
    J->mx[0] = motion0_x;
    J->my[0] = motion0_y;
    J->mx[1] = motion1_x;
    J->my[1] = motion1_y;
    J->mask[0] = mask_a;
    J->mask[1] = mask_b;
    J->interp = interp != 0;
    J->zero_origin = zero_origin != 0 || interp == 0;
    J->threshold = threshold;
    J->mode13 = mode13 != 0;
    const uint8_t *const *srcs[2] = {src0, src1};
    const int64_t *strides[2] = {src0_stride, src1_stride}, *lens[2] = {src0_len, src1_len};
    int32_t mw, mh;
    int rc = setup(*J, cfg, 2, srcs, strides, lens, src_shift, dst, dst_stride, mw, mh);
    if (rc) svpf::set_last_error("render: bad plane buffers");
    else rc = launch(*J, 1, mask_a != nullptr, mw, mh, stream);
    delete J;
    return rc;
}

int svpf_render_masked_device(const svpf_render_config *cfg, int32_t threshold, double mask_scale, int32_t mode22,
                              int32_t interp, const uint8_t *const src0[3], const int64_t src0_stride[3],
                              const int64_t src0_len[3], const uint8_t *const src1[3], const int64_t src1_stride[3],
                              const int64_t src1_len[3], int32_t src_shift, const uint16_t *motion0_x,
                              const uint16_t *motion0_y, const uint16_t *motion1_x, const uint16_t *motion1_y,
                              const uint8_t *mask_a, const uint8_t *mask_b, const uint8_t *final_mask,
                              uint8_t *const dst[3], const int64_t dst_stride[3], void *stream) {
    if (int rc = check_common(cfg, threshold, src_shift)) return rc;
    if (!src0 || !src0_stride || !src0_len || !src1 || !src1_stride || !src1_len || !dst || !dst_stride ||
        !motion0_x || !motion0_y || !motion1_x || !motion1_y || !mask_a || !mask_b) {
        svpf::set_last_error("render: null argument (masks a and b are required)");
        return SVPF_EINVAL;
    }
    if (draws_nothing(cfg)) return SVPF_OK;
    RenderJob *J = new RenderJob;
    memset(J, 0, sizeof(*J));
    J->lut_t[0] = threshold;
    J->lut_t[1] = 256 - threshold;
    J->mx[0] = motion0_x;
    J->my[0] = motion0_y;
    J->mx[1] = motion1_x;
    J->my[1] = motion1_y;
    J->mask[0] = mask_a;
    J->mask[1] = mask_b;
    J->mask[2] = final_mask;
    J->interp = interp != 0;
    J->zero_origin = interp == 0;  // render_mode21_or_22 passes zero_origin = !interp
    J->threshold = threshold;
    J->mode22 = mode22 != 0;
    {  // set_threshold_value (renderer.rs:256-264), f64 as the reference
        const double v = threshold > 126 ? 256.0 - (double)(256 - threshold) * mask_scale : (double)threshold * mask_scale;
        J->threshold_limit = as_i32(v);
    }
    const uint8_t *const *srcs[2] = {src0, src1};
    const int64_t *strides[2] = {src0_stride, src1_stride}, *lens[2] = {src0_len, src1_len};
    int32_t mw, mh;
    int rc = setup(*J, cfg, 2, srcs, strides, lens, src_shift, dst, dst_stride, mw, mh);
    if (rc) svpf::set_last_error("render: bad plane buffers");
    else rc = launch(*J, 2, final_mask != nullptr, mw, mh, stream);
    delete J;
    return rc;
}

int svpf_render_mode23_device(const svpf_render_config *cfg, int32_t threshold, int32_t interp,
                              const uint8_t *const src0[3], const int64_t src0_stride[3], const int64_t src0_len[3],
                              const uint8_t *const src1[3], const int64_t src1_stride[3], const int64_t src1_len[3],
                              int32_t src_shift, const uint16_t *const motion_x[4], const uint16_t *const motion_y[4],
                              const uint8_t *mask_a, const uint8_t *mask_b, const uint8_t *final_mask,
                              uint8_t *const dst[3], const int64_t dst_stride[3], void *stream) {
    if (int rc = check_common(cfg, threshold, src_shift)) return rc;
    bool ok = src0 && src0_stride && src0_len && src1 && src1_stride && src1_len && dst && dst_stride && motion_x &&
              motion_y && mask_a && mask_b;
    for (int k = 0; ok && k < 4; k++) ok = motion_x[k] && motion_y[k];
    if (!ok) {
        svpf::set_last_error("render: null argument (four motion sets and masks a, b are required)");
        return SVPF_EINVAL;
    }
    if (draws_nothing(cfg)) return SVPF_OK;
    RenderJob *J = new RenderJob;
    memset(J, 0, sizeof(*J));
    for (int k = 0; k < 4; k++) {  // base0, base1, next0, prev1: threshold LUT for 0 / 2, inverse for 1 / 3
        J->mx[k] = motion_x[k];
        J->my[k] = motion_y[k];
        J->lut_t[k] = (k & 1) ? 256 - threshold : threshold;
    }
    J->mask[0] = mask_a;
    J->mask[1] = mask_b;
    J->mask[2] = final_mask;
    J->interp = interp != 0;
    J->zero_origin = interp == 0;  // render_mode23 renders at zero origin when not interpolating
    J->threshold = threshold;
    const uint8_t *const *srcs[2] = {src0, src1};
    const int64_t *strides[2] = {src0_stride, src1_stride}, *lens[2] = {src0_len, src1_len};
    int32_t mw, mh;
    int rc = setup(*J, cfg, 2, srcs, strides, lens, src_shift, dst, dst_stride, mw, mh);
    if (rc) svpf::set_last_error("render: bad plane buffers");
    else rc = launch(*J, 3, final_mask != nullptr, mw, mh, stream);
    delete J;
    return rc;
}

}  // extern "C"
