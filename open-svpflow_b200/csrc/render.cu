// render.cu -- SmoothFps's single-warp frame render on the device (algorithms 1 and 2): each output
// sample is the source sample displaced by the motion interpolated between the four motion-plane
// samples around it, blended with the undisplaced sample by the mode's mask when one is given.
//
// Follows crates/svpflow-core/src/renderer.rs: CpuRenderer::render_mode1_or_2 (:308-328) through
// render_selected_warp_rows (:876-984), set_threshold (:238-250), plane_params (:1539-1606),
// motion_samples (:1608-1638), render_tiles (:1925-2010), interpolate_row / interpolate_motion
// (:2582-2637), alpha_row / alpha_at_row / alpha_at_absolute (:2639-2722), mode1_pixel (:1818-1820),
// blend_255 (:3221-3223), interp_pair (:2724-2738), interpolation_weights / coeff (:2740-2770), plane_covers /
// plane_index (:2772-2790), tile_interior (:2809-2835), sample_plane (:2837-2861), cpu_map
// (:3186-3193). The reference walks tiles (one per vector block, plus a left column and a top row
// of width / height origin) and writes each tile's samples; here one thread owns one output
// sample and finds its tile arithmetically: the last tile in the reference's loop order that
// covers the sample, since a later tile overwrites an earlier one where they overlap.
//
// 32-bit arithmetic as the reference's scalar loop. Its x86-64 SSE tile path keeps 16-bit lanes,
// which give the same values for thresholds 0..256 (|motion| <= 1024, weights <= 32), the only
// thresholds accepted here.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "../../include/svpflow_b200.h"
#include "handles.h"

namespace {

constexpr int kLut = 2048, kMaxBlock = 32;
constexpr int kPx = 4;  // output samples per thread

struct RenderPlane {
    const uint8_t *src;
    int64_t src_len, src_stride, src_span;
    uint8_t *dst;
    int64_t dst_stride;
    int32_t src_shift;
    int32_t width, height, block_w, block_h, origin_x, origin_y, x_shift, y_shift, x_div, y_div, step;
    int32_t max_x, max_y, covers;
    int32_t bw_log2, bh_log2;  // log2 of the block size when it is a power of two, else -1
    int32_t morigin_x, morigin_y;  // the plane's own origin (alpha_at_absolute's mask_params)
    int32_t xw[kMaxBlock][2], yw[kMaxBlock][2];
};

struct RenderJob {
    RenderPlane pl[3];
    const uint16_t *mx, *my;
    const uint8_t *mask;  // NULL: no mask; else grid_w x grid_h alphas (mode1_pixel blends)
    int64_t mlen;
    int32_t grid_w, grid_h, interp;
    int32_t lut_t;  // the LUT's factor: threshold (mode 2) or 256 - threshold (mode 1)
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
bool covers(const RenderPlane &p) {  // plane_covers
    if (p.src_shift != 0 && (p.src_shift >= 31 || (1 << p.src_shift) != p.step)) return false;
    const uint64_t x = (uint64_t)p.max_x, y = (uint64_t)p.max_y;
    unsigned __int128 idx;
    if (p.src_shift == 0) {
        idx = (unsigned __int128)y * (uint64_t)p.src_stride + x;
    } else {
        const uint64_t mask = (1ull << p.src_shift) - 1;
        const uint64_t sub = ((y & mask) << p.src_shift) | (x & mask);
        idx = (unsigned __int128)sub * (uint64_t)p.src_span + (unsigned __int128)(y >> p.src_shift) * (uint64_t)p.src_stride +
              (x >> p.src_shift);
    }
    return idx < (unsigned __int128)(uint64_t)p.src_len;
}

// ---- device side
__device__ __forceinline__ int64_t src_index(const RenderPlane &p, int32_t x, int32_t y) {
    if (p.src_shift == 0) return (int64_t)y * p.src_stride + x;
    const int32_t mask = (1 << p.src_shift) - 1;
    const int32_t sub = ((y & mask) << p.src_shift) | (x & mask);
    return (int64_t)sub * p.src_span + (int64_t)(y >> p.src_shift) * p.src_stride + (x >> p.src_shift);
}
__device__ __forceinline__ int32_t interp_pair(int32_t a, int32_t b, int32_t total, int32_t shift, const int32_t *w) {
    const int32_t s = (int32_t)((uint32_t)w[0] * (uint32_t)a + (uint32_t)w[1] * (uint32_t)b);
    return shift < 0 ? s / total : s >> shift;
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
__device__ __forceinline__ int32_t motion(const RenderJob &J, const uint16_t *plane, int64_t i) {
    const int k = i < J.mlen ? __ldg(plane + i) : 1024;  // NEUTRAL beyond the plane
    return ((k < kLut - 1 ? k : kLut - 1) - 1024) * J.lut_t / 256;
}

// One tile's motion (motion_samples), whether its reads are direct (plane_covers and
// tile_interior), and the motion interpolated down to row py (interpolate_motion_row).
struct TileMotion {
    int32_t rx0, rx1, ry0, ry1;
    int32_t ma0, ma1;  // the mask interpolated down to the row (alpha_row)
    bool direct;
};
__device__ __forceinline__ int32_t mask_at(const RenderJob &J, int64_t i) {
    return (i >= 0 && i < J.mlen) ? __ldg(J.mask + i) : 0;
}
__device__ __forceinline__ int32_t clamp_byte(int32_t v) { return v < 0 ? 0 : (v > 255 ? 255 : v); }
// alpha_at_absolute (renderer.rs:2687-2722): used for the mask when the motion is not interpolated
__device__ __forceinline__ int32_t alpha_absolute(const RenderJob &J, const RenderPlane &p, int32_t x, int32_t y) {
    const int32_t ox = p.morigin_x, oy = p.morigin_y, bw = p.block_w, bh = p.block_h;
    int32_t ix0 = 0, ix1 = 0, iy0 = 0, iy1 = 0;
    if (ox <= x) { ix0 = (x - ox) / bw; ix1 = ix0 + 1; }
    if (oy <= y) { iy0 = (y - oy) / bh; iy1 = iy0 + 1; }
    const int32_t fx = ox < x ? (x - ox) % bw : 0, fy = oy < y ? (y - oy) % bh : 0;
    const int64_t gw = J.grid_w;
    const int32_t tl = mask_at(J, iy0 * gw + ix0), tr = mask_at(J, iy0 * gw + ix1);
    const int32_t bl = mask_at(J, iy1 * gw + ix0), br = mask_at(J, iy1 * gw + ix1);
    const int32_t top = ((bw - fx) * tl + fx * tr) / bw, bottom = ((bw - fx) * bl + fx * br) / bw;
    return clamp_byte(((bh - fy) * top + fy * bottom) / bh);
}
__device__ __forceinline__ TileMotion tile_motion(const RenderJob &J, const RenderPlane &p, int32_t gx, int32_t bx,
                                                  int32_t tw, int32_t gy, int32_t by, int32_t th, int32_t py,
                                                  const int32_t (*syw)[2]) {
    const int64_t gw = J.grid_w;
    const int64_t i00 = (int64_t)(gy > 0 ? gy : 0) * gw + (gx > 0 ? gx : 0);
    const int64_t nx = (gx >= 0 && gx != J.grid_w - 1) ? 1 : 0, ny = (gy >= 0 && gy != J.grid_h - 1) ? gw : 0;
    int32_t sx[4], sy[4];
    const bool c = p.x_div == 2;  // chroma: motion / 2 in both axes (4:2:0)
    sx[0] = c ? motion(J, J.mx, i00) / 2 : motion(J, J.mx, i00);
    sy[0] = c ? motion(J, J.my, i00) / 2 : motion(J, J.my, i00);
    if (J.interp) {
        const int64_t ii[3] = {i00 + nx, i00 + ny, i00 + ny + nx};
#pragma unroll
        for (int q = 0; q < 3; q++) {
            sx[q + 1] = c ? motion(J, J.mx, ii[q]) / 2 : motion(J, J.mx, ii[q]);
            sy[q + 1] = c ? motion(J, J.my, ii[q]) / 2 : motion(J, J.my, ii[q]);
        }
    } else {
#pragma unroll
        for (int q = 1; q < 4; q++) { sx[q] = sx[0]; sy[q] = sy[0]; }
    }
    TileMotion t;
    t.direct = false;
    t.ma0 = t.ma1 = 0;
    if (J.mask != nullptr) {  // alpha_row
        const int32_t a = mask_at(J, i00), b = mask_at(J, i00 + nx), cc = mask_at(J, i00 + ny),
                      d = mask_at(J, i00 + ny + nx);
        if (J.interp) {
            const int32_t *wy = syw[min(py - by, kMaxBlock - 1)];
            t.ma0 = interp_pair(a, cc, p.block_h, p.y_shift, wy);
            t.ma1 = interp_pair(b, d, p.block_h, p.y_shift, wy);
        } else {
            t.ma0 = t.ma1 = a;
        }
    }
    if (p.covers && p.step > 0) {  // tile_interior over the whole tile
        int32_t mnx = sx[0], mxx = sx[0], mny = sy[0], mxy = sy[0];
#pragma unroll
        for (int q = 1; q < 4; q++) {
            mnx = min(mnx, sx[q]); mxx = max(mxx, sx[q]);
            mny = min(mny, sy[q]); mxy = max(mxy, sy[q]);
        }
        const int64_t st = p.step;
        t.direct = (int64_t)bx * st + mnx >= 0 && (int64_t)by * st + mny >= 0 &&
                   (int64_t)(bx + tw - 1) * st + mxx <= p.max_x && (int64_t)(by + th - 1) * st + mxy <= p.max_y;
    }
    if (J.interp) {
        const int32_t *wy = syw[min(py - by, kMaxBlock - 1)];
        t.rx0 = interp_pair(sx[0], sx[2], p.block_h, p.y_shift, wy);
        t.rx1 = interp_pair(sx[1], sx[3], p.block_h, p.y_shift, wy);
        t.ry0 = interp_pair(sy[0], sy[2], p.block_h, p.y_shift, wy);
        t.ry1 = interp_pair(sy[1], sy[3], p.block_h, p.y_shift, wy);
    } else {
        t.rx0 = t.rx1 = sx[0];
        t.ry0 = t.ry1 = sy[0];
    }
    return t;
}
// The source index sample (px, py) reads in its tile (interpolate_motion, then sample_plane's
// direct or clamped position).
__device__ __forceinline__ int64_t tile_sample(const RenderJob &J, const RenderPlane &p, const TileMotion &t,
                                               int32_t px, int32_t bx, int32_t py, const int32_t (*sxw)[2]) {
    int32_t dx = t.rx0, dy = t.ry0;
    if (J.interp) {
        const int32_t *wx = sxw[min(px - bx, kMaxBlock - 1)];
        dx = interp_pair(t.rx0, t.rx1, p.block_w, p.x_shift, wx);
        dy = interp_pair(t.ry0, t.ry1, p.block_w, p.x_shift, wx);
    }
    int32_t xs = px * p.step + dx, ys = py * p.step + dy;
    if (!t.direct) {
        xs = min(max(xs, 0), p.max_x);
        ys = min(max(ys, 0), p.max_y);
    }
    return src_index(p, xs, ys);
}
// With a mask: the sample's alpha (alpha_at_row, or alpha_at_absolute without interpolation)
__device__ __forceinline__ int32_t tile_alpha(const RenderJob &J, const RenderPlane &p, const TileMotion &t,
                                              int32_t px, int32_t bx, int32_t py, const int32_t (*sxw)[2]) {
    if (!J.interp) return alpha_absolute(J, p, px, py);
    return clamp_byte(interp_pair(t.ma0, t.ma1, p.block_w, p.x_shift, sxw[min(px - bx, kMaxBlock - 1)]));
}

// grid: (row length of the widest plane / (256 kPx), rows of the tallest plane, 3 planes)
template <bool MASK>
__global__ void __launch_bounds__(256) render_warp_kernel(const __grid_constant__ RenderJob J) {
    const RenderPlane &p = J.pl[blockIdx.z];
    // the plane's interpolation weights in shared memory (indexed per thread)
    __shared__ int32_t sxw[kMaxBlock][2], syw[kMaxBlock][2];
    for (int t = threadIdx.x; t < 4 * kMaxBlock; t += blockDim.x) {
        if (t < 2 * kMaxBlock) (&sxw[0][0])[t] = (&p.xw[0][0])[t];
        else (&syw[0][0])[t - 2 * kMaxBlock] = (&p.yw[0][0])[t - 2 * kMaxBlock];
    }
    __syncthreads();
    const int32_t py = blockIdx.y;
    const int32_t px0 = (blockIdx.x * blockDim.x + threadIdx.x) * kPx;
    if (px0 >= p.width || py >= p.height || p.block_w <= 0 || p.block_h <= 0) return;
    // kPx consecutive samples per thread, usually in one tile (its motion is then fetched once)
    int32_t gy, by, th;
    tile_of(py, p.origin_y, p.block_h, p.bh_log2, p.height, J.grid_h, gy, by, th);
    const int32_t pxl = min(px0 + kPx - 1, p.width - 1);
    int32_t gx, bx, tw, gxl, bxl, twl;
    tile_of(px0, p.origin_x, p.block_w, p.bw_log2, p.width, J.grid_w, gx, bx, tw);
    tile_of(pxl, p.origin_x, p.block_w, p.bw_log2, p.width, J.grid_w, gxl, bxl, twl);
    int64_t si[kPx];
    int32_t alpha[kPx];
    if (gx == gxl) {
        const TileMotion t = tile_motion(J, p, gx, bx, tw, gy, by, th, py, syw);
#pragma unroll
        for (int k = 0; k < kPx; k++) {
            si[k] = px0 + k <= pxl ? tile_sample(J, p, t, px0 + k, bx, py, sxw) : -1;
            alpha[k] = MASK && px0 + k <= pxl ? tile_alpha(J, p, t, px0 + k, bx, py, sxw) : 0;
        }
    } else {
#pragma unroll
        for (int k = 0; k < kPx; k++) {
            si[k] = -1;
            if (px0 + k > pxl) continue;
            int32_t gk, bk, twk;
            tile_of(px0 + k, p.origin_x, p.block_w, p.bw_log2, p.width, J.grid_w, gk, bk, twk);
            const TileMotion t = tile_motion(J, p, gk, bk, twk, gy, by, th, py, syw);
            si[k] = tile_sample(J, p, t, px0 + k, bk, py, sxw);
            alpha[k] = MASK ? tile_alpha(J, p, t, px0 + k, bk, py, sxw) : 0;
        }
    }
    uint8_t v[kPx];
#pragma unroll
    for (int k = 0; k < kPx; k++) v[k] = (si[k] >= 0 && si[k] < p.src_len) ? __ldg(p.src + si[k]) : (uint8_t)0;
    if (MASK) {  // mode1_pixel: blend_255(warped, base, alpha), base = the undisplaced sample
#pragma unroll
        for (int k = 0; k < kPx; k++) {
            const int64_t bi = src_index(p, (px0 + k) * p.step, py * p.step);
            const int32_t base = (px0 + k < p.width && bi >= 0 && bi < p.src_len) ? __ldg(p.src + bi) : 0;
            v[k] = (uint8_t)clamp_byte(((int32_t)v[k] * (255 - alpha[k]) + base * alpha[k] + 255) >> 8);
        }
    }
    uint8_t *out = p.dst + (int64_t)py * p.dst_stride + px0;
#pragma unroll
    for (int k = 0; k < kPx; k++)
        if (px0 + k < p.width) out[k] = v[k];
}

}  // namespace

extern "C" {

int svpf_render_warp_device(const svpf_render_config *cfg, int32_t threshold, int32_t mode1, int32_t interp,
                            const uint8_t *const src[3], const int64_t src_stride[3], const int64_t src_len[3],
                            int32_t src_shift, const uint16_t *motion_x, const uint16_t *motion_y,
                            const uint8_t *mask, uint8_t *const dst[3], const int64_t dst_stride[3], void *stream) {
    if (int rc = svpf::require_device()) return rc;
    if (!cfg || !src || !src_stride || !src_len || !dst || !dst_stride || !motion_x || !motion_y) {
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
    if (cfg->width <= 0 || cfg->height <= 0 || cfg->grid_w <= 0 || cfg->grid_h <= 0 || cfg->source_step <= 0 ||
        cfg->block_w <= 0 || cfg->block_h <= 0) {
        return SVPF_OK;  // render_tiles draws nothing
    }
    RenderJob *J = new RenderJob;
    memset(J, 0, sizeof(*J));
    // set_threshold: mode 1 warps with the inverse LUT, mode 2 with the threshold LUT
    J->lut_t = mode1 ? 256 - threshold : threshold;
    J->mx = motion_x;
    J->my = motion_y;
    J->mask = mask;
    J->mlen = (int64_t)cfg->grid_w * cfg->grid_h;
    J->grid_w = cfg->grid_w;
    J->grid_h = cfg->grid_h;
    J->interp = interp != 0;
    const int32_t cd = 2;  // SmoothFps renders 4:2:0 (CpuConfig::chroma_y_div)
    int32_t most_w = 0, most_h = 0;
    for (int pl = 0; pl < 3; pl++) {
        RenderPlane &p = J->pl[pl];
        const bool c = pl > 0;
        const bool zero = !interp;  // plane_params(chroma, zero_origin = !interp)
        p.src = src[pl];
        p.src_len = src_len[pl];
        p.src_stride = src_stride[pl];
        p.src_shift = src_shift;
        p.dst = dst[pl];
        p.dst_stride = dst_stride[pl];
        p.width = c ? cfg->width / 2 : cfg->width;
        p.height = c ? cfg->height / cd : cfg->height;
        p.src_span = p.src_stride * p.height;  // sub-planes of a super clip's level 0
        p.block_w = c ? cfg->block_w / 2 : cfg->block_w;
        p.block_h = c ? cfg->block_h / cd : cfg->block_h;
        p.origin_x = zero ? 0 : (c ? cfg->origin_x / 2 : cfg->origin_x);
        p.origin_y = zero ? 0 : (c ? cfg->origin_y / cd : cfg->origin_y);
        p.morigin_x = c ? cfg->origin_x / 2 : cfg->origin_x;
        p.morigin_y = c ? cfg->origin_y / cd : cfg->origin_y;
        p.x_shift = cpu_map(c ? cfg->block_w / 2 : cfg->block_w);
        p.y_shift = cpu_map(c ? cfg->block_h / 2 : cfg->block_h);
        p.x_div = c ? 2 : 1;
        p.y_div = c ? cd : 1;
        p.step = cfg->source_step;
        p.max_x = sat_step_max(p.width, p.step);
        p.max_y = sat_step_max(p.height, p.step);
        weights(p.block_w, p.x_shift, p.xw);
        weights(p.block_h, p.y_shift, p.yw);
        if (!p.src || !p.dst || p.src_stride < 0 || p.dst_stride < p.width || p.src_len < 0) {
            delete J;
            svpf::set_last_error("render: bad plane buffers");
            return SVPF_EINVAL;
        }
        p.covers = covers(p);
        p.bw_log2 = (p.block_w & (p.block_w - 1)) == 0 ? 31 - __builtin_clz((unsigned)p.block_w) : -1;
        p.bh_log2 = (p.block_h & (p.block_h - 1)) == 0 ? 31 - __builtin_clz((unsigned)p.block_h) : -1;
        if (p.block_w > 0 && p.block_h > 0) {
            most_w = p.width > most_w ? p.width : most_w;
            most_h = p.height > most_h ? p.height : most_h;
        }
    }
    cudaError_t e = cudaSuccess;
    if (most_w > 0 && most_h > 0) {
        dim3 grid((unsigned)((most_w + 256 * kPx - 1) / (256 * kPx)), (unsigned)most_h, 3);
        if (mask) render_warp_kernel<true><<<grid, 256, 0, (cudaStream_t)stream>>>(*J);
        else render_warp_kernel<false><<<grid, 256, 0, (cudaStream_t)stream>>>(*J);
        svpf::add_launches(1);
        e = cudaGetLastError();
    }
    delete J;
    if (e != cudaSuccess) {
        svpf::set_last_error(std::string("render: ") + cudaGetErrorString(e));
        return SVPF_ECUDA;
    }
    return SVPF_OK;
}

}  // extern "C"
