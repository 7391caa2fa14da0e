/*
 * svpf_oracle.c -- CPU restatement of open-svpflow's svpflow1 Super + Analyse path.
 *
 * TEST INFRASTRUCTURE ONLY (see svpf_oracle.h): the checker for the CUDA product,
 * and the CPU baseline that bench.py times. PARITY UNPINNED: there is no way to run
 * the Rust reference here, and it has no golden vectors; this code restates it line
 * by line and is cross-checked against an independent Python restatement.
 *
 * Rust semantics reproduced deliberately:
 *   - `usize` arithmetic wraps (release build): all usize math is done in uint64_t;
 *     `i32 as usize` sign-extends (a negative origin becomes a huge index).
 *   - `.get(i)` on a slice returns None past its length: read_or() below.
 *   - unchecked SIMD reads at a wrapped base address are emulated by the same
 *     wrapping index arithmetic, read through read_or (0 past the slice).
 *   - saturating_add / saturating_mul on u32 and i32, and `f64 as i32` (saturating,
 *     NaN -> 0), via the helpers below. The file is compiled with -fwrapv.
 *   - the reference's SSE2/AVX2 SAD/SATD equal the scalar formulas for 8-bit input
 *     (16-bit lanes never overflow: |coefficient| <= 16*255), so scalar code is used.
 * Citations: crates/svpflow1/src/{super_opts,super_build,analyse_opts,analyse_search,
 * portable,analyse_filter}.rs and crates/svpflow-core/src/params.rs.
 */
#include "svpf_oracle.h"

#include <math.h>
#include <stdbool.h>
#include <stdio.h>
#include <stdlib.h>
#include <immintrin.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef int32_t i32;
typedef int64_t i64;
typedef uint32_t u32;
typedef uint64_t u64;
typedef uint8_t u8;
typedef uint64_t usize;
typedef or_px px; /* a sample */
#ifdef OR_PX16
#define PX_MAX 1023
#define PX_MID 512
#define DC_SHIFT 2
#else
#define PX_MAX 255
#define PX_MID 128
#define DC_SHIFT 0
#endif

/* ------------------------------------------------------------------ helpers */
static inline u32 sat_add_u32(u32 a, u32 b) { u32 r = a + b; return r < a ? UINT32_MAX : r; }
static inline u32 sat_mul_u32(u32 a, u32 b) {
    u64 r = (u64)a * b;
    return r > UINT32_MAX ? UINT32_MAX : (u32)r;
}
static inline i32 sat_i64_to_i32(i64 r) {
    return r > INT32_MAX ? INT32_MAX : (r < INT32_MIN ? INT32_MIN : (i32)r);
}
static inline i32 sat_add_i32(i32 a, i32 b) { return sat_i64_to_i32((i64)a + b); }
static inline i32 sat_mul_i32(i32 a, i32 b) { return sat_i64_to_i32((i64)a * b); }
static inline usize sat_sub_us(usize a, usize b) { return a > b ? a - b : 0; }
static inline usize sat_mul_us(usize a, usize b) {
    if (a != 0 && b > UINT64_MAX / a) return UINT64_MAX;
    return a * b;
}
static inline usize sat_add_us(usize a, usize b) { usize r = a + b; return r < a ? UINT64_MAX : r; }
static inline i32 imax(i32 a, i32 b) { return a > b ? a : b; }
static inline i32 imin(i32 a, i32 b) { return a < b ? a : b; }
static inline i64 lmax(i64 a, i64 b) { return a > b ? a : b; }
static inline usize umin(usize a, usize b) { return a < b ? a : b; }
static inline i32 iclamp(i32 v, i32 lo, i32 hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline i32 f64_as_i32(double x) { /* Rust `as i32` */
    if (x != x) return 0;
    if (x >= 2147483647.0) return INT32_MAX;
    if (x <= -2147483648.0) return INT32_MIN;
    return (i32)x;
}
static inline i32 i64_as_i32(i64 v) { return (i32)(u32)(u64)v; }
static inline usize i32_as_usize(i32 v) { return (usize)(i64)v; }
static inline px avg_u8(px a, px b) { return (px)(((unsigned)a + b + 1u) >> 1); } /* super_build.rs:250 */
static inline px read_or(const px *d, usize len, usize i, px dflt) { return i < len ? d[i] : dflt; }
static inline i32 iabs(i32 v) { return v < 0 ? -v : v; }
static inline int is_blk(usize n) { return n == 4 || n == 8 || n == 16 || n == 32; }

static void set_err(char *err, size_t n, const char *msg) {
    if (err && n) { snprintf(err, n, "%s", msg); }
}

/* per-thread work counters: cost evaluations, luma px, chroma px */
/* instrumentation (not part of the reference): [0] cost evaluations, [1] luma samples and
 * [2] chroma samples compared, [3] / [4] the luma / chroma samples of [1] / [2] compared
 * under SATD. Per thread for the last pair; g_tot sums every finished pair. */
static _Thread_local u64 g_cnt[5];
static u64 g_tot[5];
void or_last_counters(uint64_t out[5]) { memcpy(out, g_cnt, sizeof(g_cnt)); }
void or_total_counters(uint64_t out[5], int32_t reset) {
    for (int i = 0; i < 5; i++) out[i] = reset ? __atomic_exchange_n(&g_tot[i], 0, __ATOMIC_RELAXED)
                                               : __atomic_load_n(&g_tot[i], __ATOMIC_RELAXED);
}
/* per level: blocks, cost evaluations, blocks that ran the bad-SAD expansion, its evaluations */
static _Thread_local u64 g_lvl[16][4];
void or_level_counters(uint64_t out[64]) { memcpy(out, g_lvl, sizeof(g_lvl)); }

/* ------------------------------------------------------------------ params lookups
 * Value::{int_at,bool_at,float_at}, crates/svpflow-core/src/params.rs:23-53 */
static const or_val k_absent = {OR_ABSENT, 0, 0.0};
static const or_val *key(const or_val *raw, int k) { return raw ? &raw[k] : &k_absent; }

static int int_at(const or_val *v, i64 *out) {
    switch (v->kind) {
    case OR_NUMBER: {
        if (!isfinite(v->num)) return 0;
        double t = trunc(v->num); /* trunc().to_string().parse::<i64>() */
        if (t >= 9223372036854775808.0 || t < -9223372036854775808.0) return 0;
        *out = (i64)t;
        return 1;
    }
    case OR_BOOL: *out = v->num != 0.0; return 1;
    case OR_NULL: *out = 0; return 1;
    default: return 0;
    }
}
static int bool_at(const or_val *v, int *out) {
    switch (v->kind) {
    case OR_NUMBER: *out = v->num != 0.0; return 1;
    case OR_STRING: case OR_OBJECT: case OR_ARRAY: *out = v->nonempty != 0; return 1;
    case OR_BOOL: *out = v->num != 0.0; return 1;
    case OR_NULL: *out = 0; return 1;
    default: return 0;
    }
}
static int float_at(const or_val *v, double *out) {
    switch (v->kind) {
    case OR_NUMBER: *out = v->num; return 1;
    case OR_BOOL: *out = v->num != 0.0 ? 1.0 : 0.0; return 1;
    case OR_NULL: *out = 0.0; return 1;
    default: return 0;
    }
}
/* opt.and_then(int_at(a)).or_else(int_at(b)).unwrap_or(d) */
static i64 int2(const or_val *raw, int a, int b, i64 d) {
    i64 t;
    if (int_at(key(raw, a), &t)) return t;
    if (b >= 0 && int_at(key(raw, b), &t)) return t;
    return d;
}
static int bool2(const or_val *raw, int a, int b, int d) {
    int t;
    if (bool_at(key(raw, a), &t)) return t;
    if (b >= 0 && bool_at(key(raw, b), &t)) return t;
    return d;
}
static double float2(const or_val *raw, int a, int b, double d) {
    double t;
    if (float_at(key(raw, a), &t)) return t;
    if (b >= 0 && float_at(key(raw, b), &t)) return t;
    return d;
}

/* ------------------------------------------------------------------ super_opts.rs */
int32_t or_reduce_dim(int32_t dim, int32_t n) { /* super_opts.rs:70-75 */
    for (i32 i = 0; i < n; i++) dim = 2 * (dim / 4);
    return dim;
}
int32_t or_auto_levels(int32_t width, int32_t height) { /* super_opts.rs:77-87 */
    for (i32 i = 0;; i++) {
        if (or_reduce_dim(height, i) < 4 || or_reduce_dim(width, i) < 4) return i;
    }
}
int32_t or_super_plane_height(int32_t base_h, int32_t pel, int32_t levels, int32_t full) {
    i32 total = full ? pel * pel * base_h : 0; /* super_opts.rs:89-95 */
    for (i32 lv = 1; lv < levels; lv++) total += or_reduce_dim(base_h, lv);
    return total;
}

int or_super_opts_from_opt(const or_val *raw, int32_t width, int32_t height, or_super_opts *o,
                           char *err, size_t err_len) { /* super_opts.rs:17-49 */
    i32 pel = i64_as_i32(int2(raw, OK_PEL, -1, 2));
    if (!(pel == 1 || pel == 2 || pel == 4)) {
        set_err(err, err_len, "SVSuper: pel has to be 1 or 2 or 4");
        return -1;
    }
    i32 gpu = i64_as_i32(int2(raw, OK_GPU, -1, 1));
    if (gpu < 0 || gpu > 2) {
        set_err(err, err_len, "SVSuper: gpu has to be 0 or 1 or 2");
        return -1;
    }
    i32 scale_down = i64_as_i32(int2(raw, OK_SCALE_DOWN, -1, 4));
    i32 scale_up = i64_as_i32(int2(raw, OK_SCALE_UP, -1, 2));
    if (gpu != 0) scale_up = 0;
    int full = bool2(raw, OK_FULL, -1, 1);
    if (pel >= 2 && !full) {
        set_err(err, err_len, "SVSuper: can't ignore finest level with high pel value");
        return -1;
    }
    int rc = bool2(raw, OK_RC, -1, 0);
    o->pel = pel; o->gpu = gpu; o->scale_down = scale_down; o->scale_up = scale_up;
    o->full = full; o->rc = rc; o->levels = or_auto_levels(width, height);
    o->width = width; o->height = height;
    return 0;
}

int64_t or_super_pack_data(const or_super_opts *o) { /* super_opts.rs:51-63 */
    u64 flags = o->rc ? 1u : 0u;
    if (!o->full) flags |= 2;
    u64 raw = (u64)(uint16_t)o->height | ((u64)(uint16_t)o->width << 16) |
              ((u64)(u8)o->pel << 32) | ((u64)(u8)o->levels << 40) | ((u64)(u8)o->gpu << 48) |
              (flags << 56);
    return (int64_t)raw;
}
int32_t or_super_height(const or_super_opts *o) {
    return or_super_plane_height(o->height, o->pel, o->levels, o->full);
}

/* ------------------------------------------------------------------ super_build.rs */
static void level_size_b(usize lv, usize luma_w, usize luma_h, int chroma, usize *w, usize *h) {
    usize yw = (usize)or_reduce_dim((i32)luma_w, (i32)lv);
    usize yh = (usize)or_reduce_dim((i32)luma_h, (i32)lv);
    if (chroma) { *w = yw / 2; *h = yh / 2; } else { *w = yw; *h = yh; }
}
static inline px sample(const px *buf, usize len, usize stride, usize row0, usize y, usize x) {
    return read_or(buf, len, (row0 + y) * stride + x, 0); /* super_build.rs:359-361 */
}

/* horizontal_6tap_inplace, super_build.rs:310-357 */
static void horizontal_6tap_inplace(px *row, usize row_len, usize dst_w, px *scratch) {
    if (dst_w == 0 || row_len == 0) return;
    if (dst_w <= 2) {
        for (usize i = 0; i < dst_w; i++) {
            px a = read_or(row, row_len, 2 * i, 0);
            px b = read_or(row, row_len, 2 * i + 1, a);
            row[i] = avg_u8(a, b);
        }
        return;
    }
    px *src = scratch;
    memcpy(src, row, row_len * sizeof(px));
    usize src_w = row_len;
    row[0] = avg_u8(src[0], read_or(src, src_w, 1, src[0]));
    px left = row[0];
    usize interior = sat_sub_us(dst_w, 2);
    for (usize i = 0; i < interior; i++) {
        usize k = 5 + 2 * i;
        px p_k = k < src_w ? src[k] : src[src_w - 1];
        px p_km3 = read_or(src, src_w, k - 3, 0);
        px p_km2 = read_or(src, src_w, k - 2, 0);
        px p_km4 = read_or(src, src_w, k - 4, 0);
        px p_even = read_or(src, src_w, (k - 1) & ~(usize)1, 0);
        u32 v = ((u32)left + p_k + 10u * ((u32)p_km3 + p_km2) + 5u * ((u32)p_km4 + p_even) + 16u) >> 5;
        row[i + 1] = (px)(v < PX_MAX ? v : PX_MAX);
        left = p_km3;
    }
    usize i = dst_w - 1 > 1 ? dst_w - 1 : 1;
    for (; i < dst_w; i++) {
        px a = read_or(src, src_w, 2 * i, 0);
        px b = read_or(src, src_w, 2 * i + 1, a);
        row[i] = avg_u8(a, b);
    }
}

/* reduce_6tap, super_build.rs:254-308 */
static void reduce_6tap(px *buf, usize len, usize stride, usize dst_row0, usize dst_w, usize dst_h,
                        usize src_row0, usize src_w, usize src_h) {
    if (dst_w == 0 || dst_h == 0 || src_w == 0 || src_h == 0) return;
    usize inter_w = src_w;
    px *inter = calloc(inter_w * dst_h, sizeof(px));
    for (usize dy = 0; dy < dst_h; dy++) {
        usize sy = dy * 2;
        i64 win0 = (i64)sy - 2;
        int use_edge = dy == 0 || dy + 1 == dst_h || win0 < 0 || (sy + 3) >= src_h;
        if (use_edge) {
            usize y0 = umin(sy, sat_sub_us(src_h, 1));
            usize y1 = umin(sy + 1, sat_sub_us(src_h, 1));
            for (usize x = 0; x < inter_w; x++) {
                px a = sample(buf, len, stride, src_row0, y0, x);
                px b = sample(buf, len, stride, src_row0, y1, x);
                inter[dy * inter_w + x] = avg_u8(a, b);
            }
        } else {
            usize st = (usize)win0;
            for (usize x = 0; x < inter_w; x++) {
                u32 p0 = sample(buf, len, stride, src_row0, st, x);
                u32 p1 = sample(buf, len, stride, src_row0, st + 1, x);
                u32 p2 = sample(buf, len, stride, src_row0, st + 2, x);
                u32 p3 = sample(buf, len, stride, src_row0, st + 3, x);
                u32 p4 = sample(buf, len, stride, src_row0, st + 4, x);
                u32 p5 = sample(buf, len, stride, src_row0, st + 5, x);
                u32 v = (p0 + p5 + 5 * (p1 + p4) + 10 * (p2 + p3) + 16) >> 5;
                inter[dy * inter_w + x] = (px)(v < PX_MAX ? v : PX_MAX);
            }
        }
    }
    px *scratch = calloc(inter_w, sizeof(px));
    for (usize dy = 0; dy < dst_h; dy++) {
        px *row = inter + dy * inter_w;
        horizontal_6tap_inplace(row, inter_w, dst_w, scratch);
        usize dst_base = (dst_row0 + dy) * stride;
        usize n = umin(inter_w, sat_sub_us(len, dst_base));
        if (n > 0) memcpy(buf + dst_base, row, n * sizeof(px));
    }
    free(scratch);
    free(inter);
}

/* fill_bilinear_pel2, super_build.rs:179-224 (in-place, sequential semantics) */
static void fill_bilinear_pel2(px *dst, usize len, usize stride, usize row0, usize w, usize h) {
    usize full = row0, hp = row0 + h, vp = row0 + 2 * h, hvp = row0 + 3 * h;
    for (usize y = 0; y < h; y++) {
        usize sb = (full + y) * stride, db = (hp + y) * stride;
        for (usize x = 0; x < w; x++) {
            px a = read_or(dst, len, sb + x, 0);
            px b = read_or(dst, len, sb + x + 1, a);
            if (db + x < len) dst[db + x] = avg_u8(a, b);
        }
    }
    for (usize y = 0; y < h; y++) {
        usize sb = (full + y) * stride, nb = (full + y + 1) * stride, db = (vp + y) * stride;
        for (usize x = 0; x < w; x++) {
            px a = read_or(dst, len, sb + x, 0);
            px b = read_or(dst, len, nb + x, a);
            if (db + x < len) dst[db + x] = avg_u8(a, b);
        }
    }
    { /* copy_row(dst, v_plane*stride, full*stride, w): memmove semantics, :226-248 */
        usize d = vp * stride, s = full * stride;
        usize n = umin(umin(w, sat_sub_us(len, d)), sat_sub_us(len, s));
        if (n && d != s) memmove(dst + d, dst + s, n * sizeof(px));
    }
    for (usize y = 0; y < h; y++) {
        usize sb = (full + y) * stride, gb = (full + y + 1) * stride + 1, db = (hvp + y) * stride;
        for (usize x = 0; x < w; x++) {
            px a = read_or(dst, len, sb + x, 0);
            px b = read_or(dst, len, gb + x, a);
            if (db + x < len) dst[db + x] = avg_u8(a, b);
        }
    }
    {
        usize d = hvp * stride, s = full * stride + 1;
        usize n = umin(umin(w, sat_sub_us(len, d)), sat_sub_us(len, s));
        if (n && d != s) memmove(dst + d, dst + s, n * sizeof(px));
    }
}

/* half(), super_build.rs:162-177; cubic8 (:138-160) computes the same value */
static px half_tap(const px *buf, usize i, usize step, usize p, usize n) {
    if (p < 2 || p + 4 >= n) return p + 1 == n ? buf[i] : avg_u8(buf[i], buf[i + step]);
    i32 value = (i32)buf[i - 2 * step] + (i32)buf[i + 3 * step] +
                5 * (4 * (i32)buf[i] - (i32)buf[i - step] + 4 * (i32)buf[i + step] - (i32)buf[i + 2 * step]) + 16;
    return (px)iclamp(value >> 5, 0, PX_MAX);
}
/* fill_bicubic_pel2 + bicubic_horizontal/vertical, super_build.rs:95-135 */
static void fill_bicubic_pel2(px *buf, usize stride, usize row0, usize w, usize h) {
    usize p0 = row0, p1 = row0 + h, p2 = row0 + 2 * h, p3 = row0 + 3 * h;
    for (usize y = 0; y < h; y++) /* horizontal full -> p1 */
        for (usize x = 0; x < w; x++) buf[(p1 + y) * stride + x] = half_tap(buf, (p0 + y) * stride + x, 1, x, w);
    for (usize y = 0; y < h; y++) /* vertical full -> p2 */
        for (usize x = 0; x < w; x++)
            buf[(p2 + y) * stride + x] = half_tap(buf, (p0 + y) * stride + x, stride, y, h);
    for (usize y = 0; y < h; y++) /* horizontal p2 -> p3 */
        for (usize x = 0; x < w; x++) buf[(p3 + y) * stride + x] = half_tap(buf, (p2 + y) * stride + x, 1, x, w);
}

/* build_plane, super_build.rs:8-93 */
void or_build_plane(px *dst, size_t dst_len, size_t dst_stride, const px *src,
                    size_t src_len, size_t src_stride, size_t src_w, size_t src_h, size_t luma_w,
                    size_t luma_h, int32_t chroma, const or_super_opts *o) {
    usize levels = (usize)(i64)o->levels, pel = (usize)(i64)o->pel;
    if (levels == 0 || src_w == 0 || src_h == 0) return;
    usize *level_y = calloc(levels, sizeof(usize));
    usize y = 0;
    for (usize lv = 0; lv < levels; lv++) {
        level_y[lv] = y;
        usize w_, h_;
        level_size_b(lv, luma_w, luma_h, chroma, &w_, &h_);
        usize sub = (lv == 0 && o->full) ? pel * pel : 1;
        y += h_ * sub;
    }
    usize base_w, base_h;
    level_size_b(0, luma_w, luma_h, chroma, &base_w, &base_h);
    {
        usize row0 = level_y[0];
        for (usize row = 0; row < umin(base_h, src_h); row++) {
            usize dst_off = (row0 + row) * dst_stride, src_off = row * src_stride;
            usize n = umin(umin(base_w, src_w), umin(sat_sub_us(dst_len, dst_off), sat_sub_us(src_len, src_off)));
            if (n > 0) memcpy(dst + dst_off, src + src_off, n * sizeof(px));
            if (base_w > 0 && dst_stride > base_w) {
                px edge = dst[dst_off + base_w - 1];
                for (usize p = base_w; p < dst_stride; p++)
                    if (dst_off + p < dst_len) dst[dst_off + p] = edge;
            }
        }
    }
    if (o->scale_down == 4) {
        for (usize lv = 0; lv + 1 < levels; lv++) {
            usize sw, sh, dw, dh;
            level_size_b(lv, luma_w, luma_h, chroma, &sw, &sh);
            level_size_b(lv + 1, luma_w, luma_h, chroma, &dw, &dh);
            reduce_6tap(dst, dst_len, dst_stride, level_y[lv + 1], dw, dh, level_y[lv], sw, sh);
        }
    }
    if (pel >= 2 && o->gpu <= 1 && o->full) {
        if (o->scale_up == 0) fill_bilinear_pel2(dst, dst_len, dst_stride, level_y[0], base_w, base_h);
        else if (o->scale_up == 2) fill_bicubic_pel2(dst, dst_stride, level_y[0], base_w, base_h);
    }
    free(level_y);
}

size_t or_super_output_len(const or_super_opts *o) {
    usize w = (usize)o->width, sh = (usize)or_super_height(o);
    return w * sh + 2 * ((w / 2) * (sh / 2));
}

void or_build_super_portable(const or_super_opts *o, const px *src, px *out) {
    usize w = (usize)o->width, h = (usize)o->height, cw = w / 2, ch = h / 2;
    usize sh = (usize)or_super_height(o);
    usize oy = w * sh, oc = cw * (sh / 2);
    memset(out, 0, (oy + 2 * oc) * sizeof(px));
    or_build_plane(out, oy, w, src, w * h, w, w, h, w, h, 0, o);
    or_build_plane(out + oy, oc, cw, src + w * h, cw * ch, cw, cw, ch, w, h, 1, o);
    or_build_plane(out + oy + oc, oc, cw, src + w * h + cw * ch, cw * ch, cw, cw, ch, w, h, 1, o);
}

void or_build_super_many(const or_super_opts *o, const px *const *src, px *const *out,
                         int32_t nframes, int32_t threads) {
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads > 0 ? threads : 1)
#endif
    for (i32 i = 0; i < nframes; i++) or_build_super_portable(o, src[i], out[i]);
    (void)threads;
}

/* ------------------------------------------------------------------ analyse_opts.rs */
int or_overlap_from_mode(int32_t bw, int32_t bh, int32_t mode, int32_t *ox, int32_t *oy, char *err,
                         size_t err_len) { /* analyse_opts.rs:259-269 */
    switch (mode) {
    case 0: *ox = 0; *oy = 0; return 0;
    case 1: *ox = bw / 8; *oy = bh / 8; return 0;
    case 2: *ox = bw / 4; *oy = bh / 4; return 0;
    case 3: *ox = bw / 2; *oy = bh / 2; return 0;
    default:
        set_err(err, err_len, "SVAnalyse: overlap must be 0, 1 (=1/8*block), 2 (=1/4*block) or 3 (=1/2*block)");
        return -1;
    }
}

int32_t or_auto_search_levels(int32_t w, int32_t h, int32_t bw, int32_t bh, int32_t ox, int32_t oy) {
    i32 sx = imax(bw - ox, 1), sy = imax(bh - oy, 1); /* analyse_opts.rs:271-295 */
    i32 gw = imax((w - ox) / sx, 0), gh = imax((h - oy) / sy, 0);
    if (gw <= 0 || gh <= 0) return 1;
    i32 end_x = ox + sx * gw, end_y = oy + sy * gh;
    i32 levels = 0;
    for (;;) {
        i32 gwl = ((end_x >> levels) - ox) / sx, ghl = ((end_y >> levels) - oy) / sy;
        if (gwl <= 0 || ghl <= 0) break;
        levels += 1;
        if (levels > 12) break;
    }
    return imax(levels, 1);
}

int or_analyse_opts_from_opt(const or_val *raw, int64_t sdata, const or_super_opts *hint,
                             or_analyse_opts *o, char *err, size_t err_len) {
    memset(o, 0, sizeof(*o));
    { /* unpack_sdata, analyse_opts.rs:243-257 */
        u64 r = (u64)sdata;
        i32 height = (i32)(r & 0xFFFF), width = (i32)((r >> 16) & 0xFFFF);
        i32 pel = (i32)((r >> 32) & 0xFF), levels = (i32)((r >> 40) & 0xFF);
        i32 selector = (i32)((r >> 48) & 0xFF);
        if (width <= 0 || height <= 0 || !(pel >= 1 && pel <= 4) || levels <= 0) {
            if (!hint) {
                set_err(err, err_len, "SVAnalyse: invalid super clip params");
                return -1;
            }
            width = hint->width; height = hint->height; pel = hint->pel; levels = hint->levels;
            selector = hint->gpu;
        }
        o->width = width; o->height = height; o->pel = pel; o->super_levels = levels;
        o->selector = selector;
    }
    i32 vectors = i64_as_i32(int2(raw, OK_VECTORS, -1, 3));
    if (vectors < 1 || vectors > 3) {
        set_err(err, err_len, "SVAnalyse: vectors must be 1, 2 or 3");
        return -1;
    }
    i32 block_w = i64_as_i32(int2(raw, OK_BLOCK_W, -1, 16));
    i32 block_h = i64_as_i32(int2(raw, OK_BLOCK_H, -1, (i64)block_w));
    if (!is_blk((usize)(i64)block_w)) {
        set_err(err, err_len, "SVAnalyse: block.w must be 4/8/16/32");
        return -1;
    }
    i32 overlap_mode = i64_as_i32(int2(raw, OK_BLOCK_OVERLAP, -1, 2));
    i32 ox, oy;
    if (or_overlap_from_mode(block_w, block_h, overlap_mode, &ox, &oy, err, err_len)) return -1;
    i32 delta = i64_as_i32(int2(raw, OK_SPECIAL_DELTA, OK_DELTA, 1));
    double lambda = float2(raw, OK_MAIN_PENALTY_LAMBDA, OK_PENALTY_LAMBDA, 10.0);
    i32 lsad = i64_as_i32(int2(raw, OK_MAIN_PENALTY_LSAD, OK_PENALTY_LSAD, 8000));
    double plevel = float2(raw, OK_MAIN_PENALTY_PLEVEL, OK_PENALTY_PLEVEL, 1.5);
    plevel = fmax(plevel, 0.01); /* f64::max ignores NaN like fmax */
    o->pnew = i64_as_i32(int2(raw, OK_MAIN_PENALTY_PNEW, OK_PENALTY_PNEW, 50));
    o->pglobal = i64_as_i32(int2(raw, OK_MAIN_PENALTY_PGLOBAL, OK_PENALTY_PGLOBAL, 50));
    o->pzero = i64_as_i32(int2(raw, OK_MAIN_PENALTY_PZERO, OK_PENALTY_PZERO, 100));
    o->pnbour = i64_as_i32(int2(raw, OK_MAIN_PENALTY_PNBOUR, OK_PENALTY_PNBOUR, 50));
    o->prev = i64_as_i32(int2(raw, OK_MAIN_PENALTY_PREV, OK_PENALTY_PREV, 0));
    i32 search_type = i64_as_i32(int2(raw, OK_MAIN_SEARCH_TYPE, OK_SEARCH_TYPE, 4));
    i32 distance = i64_as_i32(int2(raw, OK_MAIN_SEARCH_DISTANCE, OK_SEARCH_DISTANCE, 2));
    o->coarse_search_type = i64_as_i32(int2(raw, OK_MAIN_SEARCH_COARSE_TYPE, OK_SEARCH_COARSE_TYPE, (i64)search_type));
    o->coarse_distance = i64_as_i32(int2(raw, OK_MAIN_SEARCH_COARSE_DISTANCE, OK_SEARCH_COARSE_DISTANCE, 0));
    o->coarse_trymany = bool2(raw, OK_MAIN_SEARCH_COARSE_TRYMANY, OK_SEARCH_COARSE_TRYMANY, 0);
    i32 coarse_bad_sad = i64_as_i32(int2(raw, OK_MAIN_SEARCH_COARSE_BAD_SAD, OK_SEARCH_COARSE_BAD_SAD, 1000));
    o->coarse_bad_range = i64_as_i32(int2(raw, OK_MAIN_SEARCH_COARSE_BAD_RANGE, -1, -24));
    o->fine_satd = bool2(raw, OK_MAIN_SEARCH_SATD, OK_SEARCH_SATD, 0);
    o->coarse_satd = bool2(raw, OK_MAIN_SEARCH_COARSE_SATD, -1, 1);
    o->sort = bool2(raw, OK_MAIN_SEARCH_SORT, OK_SORT, 1);
    /* refine = opt.array_at(["refine"]).first(), analyse_opts.rs:150-164 */
    int has_refine = key(raw, OK_REFINE0)->kind != OR_ABSENT;
    i64 t;
    o->has_refine_thsad = 0;
    if (has_refine && int_at(key(raw, OK_REFINE0_THSAD), &t)) {
        o->has_refine_thsad = 1;
        o->refine_thsad = i64_as_i32(t) * imax((block_w / 2) * (block_h / 2), 1) / 32;
    }
    o->refine_search_type = has_refine ? i64_as_i32(int2(raw, OK_REFINE0_SEARCH_TYPE, -1, (i64)search_type)) : search_type;
    o->refine_distance = has_refine ? i64_as_i32(int2(raw, OK_REFINE0_SEARCH_DISTANCE, -1, (i64)distance)) : distance;
    o->refine_satd = has_refine ? bool2(raw, OK_REFINE0_SEARCH_SATD, -1, o->fine_satd) : o->fine_satd;

    i32 levels = imax(imin(or_auto_search_levels(o->width, o->height, block_w, block_h, ox, oy), o->super_levels), 1);
    if (int_at(key(raw, OK_MAIN_LEVELS), &t) && t > 0) levels = imax(imin(i64_as_i32(t), o->super_levels), 1);

    double area = (double)imax(block_w * block_h, 1);
    o->lambda = f64_as_i32(2.0 * area * 1000.0 * 0.015625 * lambda);
    i32 area_scale = imax(block_w * block_h, 1) / 32;
    o->lsad = sat_mul_i32(lsad, area_scale);
    o->coarse_bad_sad = sat_mul_i32(coarse_bad_sad, area_scale);

    o->vectors = vectors; o->block_w = block_w; o->block_h = block_h; o->overlap_mode = overlap_mode;
    o->overlap_x = ox; o->overlap_y = oy; o->delta = delta; o->levels = levels; o->plevel = plevel;
    o->search_type = search_type; o->distance = distance;
    return 0;
}

int or_analyser_portable(const or_super_opts *so, int32_t bw, int32_t bh, int32_t overlap_mode,
                         int32_t vectors, or_analyse_opts *o, char *err, size_t err_len) {
    if (!is_blk((usize)(i64)bw) || !is_blk((usize)(i64)bh)) { /* portable.rs:189-229 */
        set_err(err, err_len, "block dimensions must be 4, 8, 16 or 32");
        return -1;
    }
    if (vectors < 1 || vectors > 3) {
        set_err(err, err_len, "vectors must be 1, 2 or 3");
        return -1;
    }
    i32 ox, oy;
    if (or_overlap_from_mode(bw, bh, overlap_mode, &ox, &oy, err, err_len)) return -1;
    if (or_analyse_opts_from_opt(NULL, or_super_pack_data(so), so, o, err, err_len)) return -1;
    o->vectors = vectors; o->block_w = bw; o->block_h = bh; o->overlap_mode = overlap_mode;
    o->overlap_x = ox; o->overlap_y = oy;
    o->levels = imax(imin(or_auto_search_levels(o->width, o->height, bw, bh, ox, oy), o->super_levels), 1);
    o->lambda = f64_as_i32((double)(bw * bh) * 312.5);
    return 0;
}

void or_output_block(const or_analyse_opts *o, int32_t *bw, int32_t *bh, int32_t *ox, int32_t *oy) {
    if (o->has_refine_thsad) { /* analyse_opts.rs:221-232 */
        *bw = imax(o->block_w / 2, 4); *bh = imax(o->block_h / 2, 4);
        *ox = imax(o->overlap_x / 2, 0); *oy = imax(o->overlap_y / 2, 0);
    } else {
        *bw = o->block_w; *bh = o->block_h; *ox = o->overlap_x; *oy = o->overlap_y;
    }
}
void or_grid(const or_analyse_opts *o, int32_t bw, int32_t bh, int32_t ox, int32_t oy, int32_t *gw,
             int32_t *gh) { /* analyse_opts.rs:234-240 */
    i32 sx = imax(bw - ox, 1), sy = imax(bh - oy, 1);
    *gw = imax((o->width - ox) / sx, 1);
    *gh = imax((o->height - oy) / sy, 1);
}
void or_level_grid(const or_analyse_opts *o, int32_t level, int32_t *gw_out, int32_t *gh_out) {
    i32 bw = o->block_w, bh = o->block_h, ox = o->overlap_x, oy = o->overlap_y; /* :1453-1463 */
    i32 step_x = imax(bw - ox, 1), step_y = imax(bh - oy, 1);
    i32 gw0 = imax((o->width - ox) / step_x, 0), gh0 = imax((o->height - oy) / step_y, 0);
    i32 end_x = ox + step_x * gw0, end_y = oy + step_y * gh0;
    i32 gw = imax(((end_x >> level) - ox) / step_x, 1), gh = imax(((end_y >> level) - oy) / step_y, 1);
    *gw_out = gw + (level > 0);
    *gh_out = gh + (level > 0);
}

/* ------------------------------------------------------------------ analyse_search.rs */
typedef struct { i32 x, y; } pt;
typedef struct { pt mv; u32 sad; i64 cost; } best_t; /* SearchBest, :228-233 */
typedef struct { i32 min_x, min_y, max_x, max_y; } bounds_t;

static usize level_y_offset(const or_planes *p, i32 level) { /* :49-58 */
    usize y = 0, pel = (usize)(i64)p->pel;
    for (i32 lv = 0; lv < level; lv++) {
        usize h = (usize)(i64)or_reduce_dim((i32)p->luma_h, lv);
        usize sub = (lv == 0 && p->full) ? pel * pel : 1;
        y += h * sub;
    }
    return y;
}
static void level_size(const or_planes *p, i32 level, usize *w, usize *h) { /* :60-65 */
    *w = (usize)(i64)or_reduce_dim((i32)p->luma_w, level);
    *h = (usize)(i64)or_reduce_dim((i32)p->luma_h, level);
}
static usize chroma_level_offset(const or_planes *p, i32 level) { /* :2704-2713 */
    usize y = 0, pel = (usize)(i64)p->pel;
    for (i32 lv = 0; lv < level; lv++) {
        usize h = (usize)(i64)or_reduce_dim((i32)p->luma_h, lv) / 2;
        usize sub = (lv == 0 && p->full) ? pel * pel : 1;
        y += (h > 1 ? h : 1) * sub;
    }
    return y;
}

uint32_t or_hadamard4_satd(const int32_t d[16]) { /* hadamard4_satd, :2681-2702 */
    i32 t[4][4];
    for (int i = 0; i < 4; i++) {
        i32 s0 = d[i * 4 + 0] + d[i * 4 + 1], s1 = d[i * 4 + 0] - d[i * 4 + 1];
        i32 s2 = d[i * 4 + 2] + d[i * 4 + 3], s3 = d[i * 4 + 2] - d[i * 4 + 3];
        t[i][0] = s0 + s2; t[i][1] = s1 + s3; t[i][2] = s0 - s2; t[i][3] = s1 - s3;
    }
    i32 s = 0;
    for (int j = 0; j < 4; j++) {
        i32 s0 = t[0][j] + t[1][j], s1 = t[0][j] - t[1][j];
        i32 s2 = t[2][j] + t[3][j], s3 = t[2][j] - t[3][j];
        s += iabs(s0 + s2) + iabs(s1 + s3) + iabs(s0 - s2) + iabs(s1 - s3);
    }
    return (u32)(s > 0 ? s : 0);
}

/* Vector forms of the interior SAD / SATD for blocks whose every byte is in its slice, as
 * the reference's own sad_u8_simd (:1857-1994) and hadamard4_satd_sse2/avx2 (:2523-2679)
 * are: the same sums, in 16-bit lanes (|coefficient| <= 16 * 255 never overflows). Used by
 * the CPU baseline's speed only; the scalar forms below remain the definition. */
#ifndef OR_PX16
static int in_slice(usize len, usize i, usize stride, usize w, usize h) {
    if (i > len || h == 0) return 0;
    usize rest = len - i;
    if (h - 1 > 0 && stride > (rest - (w <= rest ? w : rest)) / (h - 1)) return 0;
    return (h - 1) * stride + w <= rest;
}
static inline u32 sad_row_simd(const u8 *a, const u8 *b, usize w) {
    if (w == 32) {
        __m256i d = _mm256_sad_epu8(_mm256_loadu_si256((const __m256i *)a), _mm256_loadu_si256((const __m256i *)b));
        __m128i t = _mm_add_epi64(_mm256_castsi256_si128(d), _mm256_extracti128_si256(d, 1));
        return (u32)(_mm_cvtsi128_si32(t) + _mm_extract_epi32(t, 2));
    }
    if (w == 16) {
        __m128i d = _mm_sad_epu8(_mm_loadu_si128((const __m128i *)a), _mm_loadu_si128((const __m128i *)b));
        return (u32)(_mm_cvtsi128_si32(d) + _mm_extract_epi32(d, 2));
    }
    u64 x = 0, y = 0;
    memcpy(&x, a, w);
    memcpy(&y, b, w);
    return (u32)_mm_cvtsi128_si32(_mm_sad_epu8(_mm_cvtsi64_si128((long long)x), _mm_cvtsi64_si128((long long)y)));
}
/* sum of |H4 D H4| over the 4x4 tiles of a 4-row strip, 16 columns (4 tiles) at a time */
static inline __m256i satd_strip16(const u8 *a, usize as, const u8 *b, usize bs) {
    __m256i d[4];
    for (int r = 0; r < 4; r++)
        d[r] = _mm256_sub_epi16(_mm256_cvtepu8_epi16(_mm_loadu_si128((const __m128i *)(a + r * as))),
                                _mm256_cvtepu8_epi16(_mm_loadu_si128((const __m128i *)(b + r * bs))));
    __m256i s0 = _mm256_add_epi16(d[0], d[1]), s1 = _mm256_sub_epi16(d[0], d[1]);
    __m256i s2 = _mm256_add_epi16(d[2], d[3]), s3 = _mm256_sub_epi16(d[2], d[3]);
    __m256i v[4] = {_mm256_add_epi16(s0, s2), _mm256_add_epi16(s1, s3), _mm256_sub_epi16(s0, s2),
                    _mm256_sub_epi16(s1, s3)};
    __m256i acc = _mm256_setzero_si256();
    const __m256i ones = _mm256_set1_epi16(1);
    for (int k = 0; k < 4; k++) { /* horizontal 4-point transform inside each group of 4 lanes */
        __m256i x = v[k];
        __m256i sw = _mm256_shufflehi_epi16(_mm256_shufflelo_epi16(x, 0xB1), 0xB1); /* 1 0 3 2 */
        __m256i t = _mm256_blend_epi16(_mm256_add_epi16(x, sw), _mm256_sub_epi16(sw, x), 0xAA);
        __m256i sw2 = _mm256_shufflehi_epi16(_mm256_shufflelo_epi16(t, 0x4E), 0x4E); /* 2 3 0 1 */
        __m256i u = _mm256_blend_epi16(_mm256_add_epi16(t, sw2), _mm256_sub_epi16(sw2, t), 0xCC);
        acc = _mm256_add_epi32(acc, _mm256_madd_epi16(_mm256_abs_epi16(u), ones));
    }
    return acc;
}
static inline u32 hsum_epi32(__m256i v) {
    __m128i t = _mm_add_epi32(_mm256_castsi256_si128(v), _mm256_extracti128_si256(v, 1));
    t = _mm_add_epi32(t, _mm_shuffle_epi32(t, 0x4E));
    t = _mm_add_epi32(t, _mm_shuffle_epi32(t, 0xB1));
    return (u32)_mm_cvtsi128_si32(t);
}

#endif

/* sad_u8_simd (:1857-1951): plain sum of |a-b| at (possibly wrapped) base indices */
static u32 sad_raw(const px *a, usize alen, usize ai, usize as, const px *b, usize blen, usize bi,
                   usize bs, usize w, usize h) {
#ifndef OR_PX16
    if ((w == 4 || w == 8 || w == 16 || w == 32) && in_slice(alen, ai, as, w, h) && in_slice(blen, bi, bs, w, h)) {
        u32 t = 0;
        for (usize r = 0; r < h; r++) t += sad_row_simd(a + ai + r * as, b + bi + r * bs, w);
        return t;
    }
#endif
    u32 s = 0;
    for (usize r = 0; r < h; r++)
        for (usize c = 0; c < w; c++) {
            i32 x = read_or(a, alen, ai + r * as + c, 0), y = read_or(b, blen, bi + r * bs + c, 0);
            s += (u32)iabs(x - y);
        }
    return s;
}
/* satd_interior (:2439-2521) == (sum of per-tile hadamard4_satd) >> 1 */
static u32 satd_raw(const px *a, usize alen, usize ai, usize as, const px *b, usize blen, usize bi,
                    usize bs, usize n) {
#ifndef OR_PX16
    if ((n == 16 || n == 32) && in_slice(alen, ai, as, n, n) && in_slice(blen, bi, bs, n, n)) {
        __m256i acc = _mm256_setzero_si256();
        for (usize ty = 0; ty < n; ty += 4)
            for (usize tx = 0; tx < n; tx += 16)
                acc = _mm256_add_epi32(acc, satd_strip16(a + ai + ty * as + tx, as, b + bi + ty * bs + tx, bs));
        return hsum_epi32(acc) >> 1;
    }
#endif
    u32 total = 0;
    usize tiles = n / 4;
    for (usize ty = 0; ty < tiles; ty++)
        for (usize tx = 0; tx < tiles; tx++) {
            i32 d[16];
            for (usize r = 0; r < 4; r++)
                for (usize c = 0; c < 4; c++)
                    d[r * 4 + c] = (i32)read_or(a, alen, ai + (ty * 4 + r) * as + tx * 4 + c, 0) -
                                   (i32)read_or(b, blen, bi + (ty * 4 + r) * bs + tx * 4 + c, 0);
            total = sat_add_u32(total, or_hadamard4_satd(d));
        }
    return total >> 1;
}

static bounds_t mv_bounds(i32 px, i32 py, i32 bw, i32 bh, i32 lw, i32 lh, i32 pel) { /* :1619-1636 */
    pel = imax(pel, 1);
    bounds_t b = {-pel * px, -pel * py, pel * (lw - px - bw) + 1, pel * (lh - py - bh) + 1};
    return b;
}
/* edge_shift_origins, :1638-1676; returns 0 for None */
static int edge_shift_origins(i32 px, i32 py, i32 mvx, i32 mvy, i32 bw, i32 bh, i32 lw, i32 lh, i32 pel,
                              i32 *cx_o, i32 *cy_o, i32 *rx_o, i32 *ry_o) {
    pel = imax(pel, 1);
    bounds_t b = mv_bounds(px, py, bw, bh, lw, lh, pel);
    i32 ox = mvx < b.min_x ? mvx - b.min_x : ((b.max_x > b.min_x && mvx >= b.max_x) ? mvx + 1 - b.max_x : 0);
    i32 oy = mvy < b.min_y ? mvy - b.min_y : ((b.max_y > b.min_y && mvy >= b.max_y) ? mvy + 1 - b.max_y : 0);
    if (ox == 0 && oy == 0) return 0;
    i32 cx = iclamp(px - ox, 0, imax(lw - bw, 0)), cy = iclamp(py - oy, 0, imax(lh - bh, 0));
    i32 rx, ry;
    if (pel == 1) { rx = cx + mvx; ry = cy + mvy; }
    else if (pel == 4) { rx = (4 * cx + mvx) >> 2; ry = (4 * cy + mvy) >> 2; }
    else { rx = (2 * cx + mvx) >> 1; ry = (2 * cy + mvy) >> 1; }
    *cx_o = cx; *cy_o = cy; *rx_o = rx; *ry_o = ry;
    return 1;
}

/* satd_edge, :2305-2351 */
static u32 satd_edge(const px *s, usize slen, usize sstride, usize srow, i32 sx0, i32 sy0, const px *r,
                     usize rlen, usize rstride, usize rrow, i32 rx0, i32 ry0, usize width, usize height,
                     usize n) {
    i32 w = (i32)width, h = (i32)height;
    u32 total = 0;
    usize tiles = n / 4;
    for (usize ty = 0; ty < tiles; ty++)
        for (usize tx = 0; tx < tiles; tx++) {
            i32 d[16];
            for (usize rr = 0; rr < 4; rr++) {
                usize sy = (usize)iclamp(sy0 + (i32)(ty * 4 + rr), 0, imax(h - 1, 0));
                usize ry = (usize)iclamp(ry0 + (i32)(ty * 4 + rr), 0, imax(h - 1, 0));
                for (usize c = 0; c < 4; c++) {
                    usize sx = (usize)iclamp(sx0 + (i32)(tx * 4 + c), 0, imax(w - 1, 0));
                    usize rx = (usize)iclamp(rx0 + (i32)(tx * 4 + c), 0, imax(w - 1, 0));
                    i32 a = read_or(s, slen, (srow + sy) * sstride + sx, 0);
                    i32 b = read_or(r, rlen, (rrow + ry) * rstride + rx, 0);
                    d[rr * 4 + c] = a - b;
                }
            }
            total = sat_add_u32(total, or_hadamard4_satd(d));
        }
    return total >> 1;
}

/* satd_luma_clamp, :2353-2436 */
static u32 satd_luma_clamp(const or_planes *src, const or_planes *ref, usize cur_row0, usize ref_row0,
                           usize px, usize py, i32 mv_x, i32 mv_y, usize lw, usize lh, usize n) {
    i32 rx0 = (i32)px + mv_x, ry0 = (i32)py + mv_y;
    usize src_end = sat_add_us(sat_mul_us(cur_row0 + py + n - 1, src->y_stride), px + n);
    usize ref_end = ry0 >= 0
        ? sat_add_us(sat_mul_us(ref_row0 + (usize)ry0 + n - 1, ref->y_stride), (usize)imax(rx0, 0) + n)
        : UINT64_MAX;
    int interior = px + n <= lw && py + n <= lh && rx0 >= 0 && ry0 >= 0 && (usize)rx0 + n <= lw &&
                   (usize)ry0 + n <= lh && src_end <= src->y_len && ref_end <= ref->y_len;
    if (interior) {
        usize si = (cur_row0 + py) * src->y_stride + px;
        usize ri = (ref_row0 + (usize)ry0) * ref->y_stride + (usize)rx0;
        return satd_raw(src->y, src->y_len, si, src->y_stride, ref->y, ref->y_len, ri, ref->y_stride, n);
    }
    u32 total = 0;
    usize tiles = n / 4;
    for (usize ty = 0; ty < tiles; ty++)
        for (usize tx = 0; tx < tiles; tx++) {
            i32 d[16];
            for (usize r = 0; r < 4; r++) {
                usize sy = py + ty * 4 + r;
                usize ry = (usize)iclamp((i32)py + (i32)(ty * 4 + r) + mv_y, 0, (i32)lh - 1);
                for (usize c = 0; c < 4; c++) {
                    usize sx = px + tx * 4 + c;
                    usize rx = (usize)iclamp((i32)px + (i32)(tx * 4 + c) + mv_x, 0, (i32)lw - 1);
                    i32 a = (sy < lh && sx < lw) ? read_or(src->y, src->y_len, (cur_row0 + sy) * src->y_stride + sx, 0) : 0;
                    i32 b = read_or(ref->y, ref->y_len, (ref_row0 + ry) * ref->y_stride + rx, 0);
                    d[r * 4 + c] = a - b;
                }
            }
            total = sat_add_u32(total, or_hadamard4_satd(d));
        }
    return total >> 1;
}

/* block_cost_luma_interior, :1719-1852 (compute_luma is false at every call site) */
static u32 luma_interior(const or_planes *src, const or_planes *ref, i32 level, i32 px, i32 py, usize bw,
                         usize bh, i32 mvx, i32 mvy, int use_satd, i32 pel) {
    usize lw, lh;
    level_size(src, level, &lw, &lh);
    px = px - (level > 0 && px + (i32)bw >= (i32)lw);
    py = py - (level > 0 && py + (i32)bh >= (i32)lh);
    usize px_u = i32_as_usize(px), py_u = i32_as_usize(py);
    usize y_off = level_y_offset(src, level);
    i32 sub_x = 0, sub_y = 0, mx = mvx, my = mvy;
    if (level == 0 && pel >= 2) { sub_x = mvx & 1; sub_y = mvy & 1; mx = mvx >> 1; my = mvy >> 1; }
    usize sub_idx = i32_as_usize(sub_y * pel + sub_x);
    usize cur_row0 = y_off, ref_row0 = y_off + sub_idx * lh;
    g_cnt[1] += bw * bh;
    if (use_satd && is_blk(bw) && is_blk(bh) && bw == bh) {
        g_cnt[3] += bw * bh;
        return satd_luma_clamp(src, ref, cur_row0, ref_row0, px_u, py_u, mx, my, lw, lh, bw);
    }
    i32 rx0 = px + mx, ry0 = py + my;
    int interior = px >= 0 && py >= 0 && rx0 >= 0 && ry0 >= 0 && (usize)px + bw <= lw &&
                   (usize)py + bh <= lh && (usize)rx0 + bw <= lw && (usize)ry0 + bh <= lh;
    if (interior && is_blk(bw)) {
        usize si = (cur_row0 + py_u) * src->y_stride + px_u;
        usize ri = (ref_row0 + (usize)ry0) * ref->y_stride + (usize)rx0;
        return sad_raw(src->y, src->y_len, si, src->y_stride, ref->y, ref->y_len, ri, ref->y_stride, bw, bh);
    }
    u32 sad = 0;
    for (usize row = 0; row < bh; row++) {
        usize sy = py_u + row;
        usize ry = (usize)iclamp(py + (i32)row + my, 0, (i32)lh - 1);
        if (sy >= lh) break;
        for (usize col = 0; col < bw; col++) {
            usize sx = px_u + col;
            usize rx = (usize)iclamp(px + (i32)col + mx, 0, (i32)lw - 1);
            if (sx >= lw) break;
            i32 a = read_or(src->y, src->y_len, (cur_row0 + sy) * src->y_stride + sx, 0);
            i32 b = read_or(ref->y, ref->y_len, (ref_row0 + ry) * ref->y_stride + rx, 0);
            sad = sat_add_u32(sad, (u32)iabs(a - b));
        }
    }
    return sad;
}

/* chroma_sad_x4, :2169-2303 */
static u32 chroma_sad_x4(const or_planes *src, const or_planes *ref, i32 level, i32 pel, i32 mvx, i32 mvy,
                         usize px, usize py, usize bw, usize bh, usize lw, usize lh, int use_satd) {
    usize cw = bw / 2, ch = bh / 2;
    if (cw < 4 || ch < 4) return 0;
    g_cnt[2] += 2 * cw * ch;
    usize cpx = px / 2, cpy = py / 2, clw = lw / 2, clh = lh / 2;
    usize c_off = chroma_level_offset(src, level);
    usize c_sub_idx = 0;
    i32 mv_cx, mv_cy;
    if (level == 0 && pel >= 2) {
        c_sub_idx = i32_as_usize((mvy & 1) * pel + (mvx & 1));
        mv_cx = mvx >> 2; mv_cy = mvy >> 2;
    } else { mv_cx = mvx >> 1; mv_cy = mvy >> 1; }
    usize c_cur = c_off;
    usize c_ref = c_off + ((level == 0 && pel > 1) ? c_sub_idx * clh : 0);
    if (cw == 4 || cw == 8 || cw == 16) {
        i32 rx0 = (i32)cpx + mv_cx, ry0 = (i32)cpy + mv_cy;
        if (cpx + cw <= clw && cpy + ch <= clh && rx0 >= 0 && ry0 >= 0 && (usize)rx0 + cw <= clw &&
            (usize)ry0 + ch <= clh) {
            usize su = (c_cur + cpy) * src->u_stride + cpx, sv = (c_cur + cpy) * src->v_stride + cpx;
            usize ru = (c_ref + (usize)ry0) * ref->u_stride + (usize)rx0;
            usize rv = (c_ref + (usize)ry0) * ref->v_stride + (usize)rx0;
            if (su + (ch - 1) * src->u_stride + cw <= src->u_len && sv + (ch - 1) * src->v_stride + cw <= src->v_len &&
                ru + (ch - 1) * ref->u_stride + cw <= ref->u_len && rv + (ch - 1) * ref->v_stride + cw <= ref->v_len) {
                u32 a, b;
                if (use_satd) { /* satd_interior(.., cw): an n x n square with n = cw */
                    g_cnt[4] += 2 * cw * cw;
                    a = satd_raw(src->u, src->u_len, su, src->u_stride, ref->u, ref->u_len, ru, ref->u_stride, cw);
                    b = satd_raw(src->v, src->v_len, sv, src->v_stride, ref->v, ref->v_len, rv, ref->v_stride, cw);
                } else {
                    a = sad_raw(src->u, src->u_len, su, src->u_stride, ref->u, ref->u_len, ru, ref->u_stride, cw, ch);
                    b = sad_raw(src->v, src->v_len, sv, src->v_stride, ref->v, ref->v_len, rv, ref->v_stride, cw, ch);
                }
                return sat_mul_u32(sat_add_u32(a, b), 4);
            }
        }
    }
    u32 sad_uv = 0;
    for (usize row = 0; row < ch; row++) {
        usize sy = cpy + row;
        usize ry = (usize)iclamp((i32)cpy + (i32)row + mv_cy, 0, (i32)clh - 1);
        if (sy >= clh) break;
        for (usize col = 0; col < cw; col++) {
            usize sx = cpx + col;
            usize rx = (usize)iclamp((i32)cpx + (i32)col + mv_cx, 0, (i32)clw - 1);
            if (sx >= clw) break;
            i32 au = read_or(src->u, src->u_len, (c_cur + sy) * src->u_stride + sx, PX_MID);
            i32 av = read_or(src->v, src->v_len, (c_cur + sy) * src->v_stride + sx, PX_MID);
            i32 bu = read_or(ref->u, ref->u_len, (c_ref + ry) * ref->u_stride + rx, PX_MID);
            i32 bv = read_or(ref->v, ref->v_len, (c_ref + ry) * ref->v_stride + rx, PX_MID);
            sad_uv = sat_add_u32(sat_add_u32(sad_uv, (u32)iabs(au - bu)), (u32)iabs(av - bv));
        }
    }
    return sat_mul_u32(sad_uv, 4);
}

/* block_cost_edge_lc, :1996-2167; returns 0 for None */
static int block_cost_edge_lc(const or_planes *src, const or_planes *ref, i32 level, i32 px, i32 py, i32 bw,
                              i32 bh, i32 mvx, i32 mvy, int use_satd, i32 pel, u32 *lo, u32 *co) {
    usize lw, lh;
    level_size(src, level, &lw, &lh);
    i32 cx, cy, rx0, ry0;
    if (!edge_shift_origins(px, py, mvx, mvy, bw, bh, (i32)lw, (i32)lh, pel, &cx, &cy, &rx0, &ry0)) return 0;
    usize y_off = level_y_offset(src, level);
    i32 sub_x = 0, sub_y = 0;
    if (level == 0 && pel >= 2) { sub_x = mvx & 1; sub_y = mvy & 1; }
    usize sub_idx = i32_as_usize(sub_y * pel + sub_x);
    usize cur_row0 = y_off, ref_row0 = y_off + sub_idx * lh;
    usize bw_u = i32_as_usize(bw), bh_u = i32_as_usize(bh);
    i32 lw_i = (i32)lw, lh_i = (i32)lh;
    u32 sad_l;
    g_cnt[1] += bw_u * bh_u;
    if (use_satd && is_blk(bw_u) && is_blk(bh_u) && bw_u == bh_u) {
        g_cnt[3] += bw_u * bh_u;
        sad_l = satd_edge(src->y, src->y_len, src->y_stride, cur_row0, cx, cy, ref->y, ref->y_len, ref->y_stride,
                          ref_row0, rx0, ry0, lw, lh, bw_u);
    } else {
        u32 sad = 0;
        for (usize row = 0; row < bh_u; row++) {
            usize sy = (usize)iclamp(cy + (i32)row, 0, imax(lh_i - 1, 0));
            usize ry = (usize)iclamp(ry0 + (i32)row, 0, imax(lh_i - 1, 0));
            for (usize col = 0; col < bw_u; col++) {
                usize sx = (usize)iclamp(cx + (i32)col, 0, imax(lw_i - 1, 0));
                usize rx = (usize)iclamp(rx0 + (i32)col, 0, imax(lw_i - 1, 0));
                i32 a = read_or(src->y, src->y_len, (cur_row0 + sy) * src->y_stride + sx, 0);
                i32 b = read_or(ref->y, ref->y_len, (ref_row0 + ry) * ref->y_stride + rx, 0);
                sad = sat_add_u32(sad, (u32)iabs(a - b));
            }
        }
        sad_l = sad;
    }
    usize cw = bw_u / 2, ch = bh_u / 2, clw = lw / 2, clh = lh / 2;
    i32 ccx = (px >> 1) - ((px - cx) >> 1), ccy = (py >> 1) - ((py - cy) >> 1); /* :1679-1681 */
    i32 crx0 = ((mvx >> 1) + 2 * ccx) >> 1, cry0 = ((mvy >> 1) + 2 * ccy) >> 1;
    usize c_off = chroma_level_offset(src, level);
    usize c_sub = (level == 0 && pel >= 2) ? i32_as_usize((mvy & 1) * pel + (mvx & 1)) : 0;
    usize c_ref = c_off + c_sub * clh;
    i32 clw_i = (i32)clw, clh_i = (i32)clh;
    u32 sad_uv;
    g_cnt[2] += 2 * cw * ch;
    if (use_satd && cw == ch && (cw == 4 || cw == 8 || cw == 16)) {
        g_cnt[4] += 2 * cw * ch;
        sad_uv = sat_add_u32(
            satd_edge(src->u, src->u_len, src->u_stride, c_off, ccx, ccy, ref->u, ref->u_len, ref->u_stride, c_ref,
                      crx0, cry0, clw, clh, cw),
            satd_edge(src->v, src->v_len, src->v_stride, c_off, ccx, ccy, ref->v, ref->v_len, ref->v_stride, c_ref,
                      crx0, cry0, clw, clh, cw));
    } else {
        u32 sad = 0;
        for (usize row = 0; row < ch; row++) {
            usize sy = (usize)iclamp(ccy + (i32)row, 0, imax(clh_i - 1, 0));
            usize ry = (usize)iclamp(cry0 + (i32)row, 0, imax(clh_i - 1, 0));
            for (usize col = 0; col < cw; col++) {
                usize sx = (usize)iclamp(ccx + (i32)col, 0, imax(clw_i - 1, 0));
                usize rx = (usize)iclamp(crx0 + (i32)col, 0, imax(clw_i - 1, 0));
                i32 au = read_or(src->u, src->u_len, (c_off + sy) * src->u_stride + sx, PX_MID);
                i32 bu = read_or(ref->u, ref->u_len, (c_ref + ry) * ref->u_stride + rx, PX_MID);
                i32 av = read_or(src->v, src->v_len, (c_off + sy) * src->v_stride + sx, PX_MID);
                i32 bv = read_or(ref->v, ref->v_len, (c_ref + ry) * ref->v_stride + rx, PX_MID);
                sad = sat_add_u32(sat_add_u32(sad, (u32)iabs(au - bu)), (u32)iabs(av - bv));
            }
        }
        sad_uv = sad;
    }
    *lo = sad_l;
    *co = sat_mul_u32(sad_uv, 4);
    return 1;
}

/* block_cost_lc, :1683-1717 */
static void block_cost_lc(const or_planes *src, const or_planes *ref, i32 level, i32 px, i32 py, i32 bw, i32 bh,
                          i32 mvx, i32 mvy, int use_satd, i32 pel, u32 *l, u32 *c) {
    pel = imax(pel, 1);
    usize lw, lh;
    level_size(src, level, &lw, &lh);
    g_cnt[0]++;
    if (block_cost_edge_lc(src, ref, level, px, py, bw, bh, mvx, mvy, use_satd, pel, l, c)) return;
    *l = luma_interior(src, ref, level, px, py, i32_as_usize(bw), i32_as_usize(bh), mvx, mvy, use_satd, pel);
    *c = chroma_sad_x4(src, ref, level, pel, mvx, mvy, i32_as_usize(px), i32_as_usize(py), i32_as_usize(bw),
                       i32_as_usize(bh), lw, lh, use_satd);
}
void or_block_cost_lc(const or_planes *src, const or_planes *ref, int32_t level, int32_t px, int32_t py,
                      int32_t bw, int32_t bh, int32_t mvx, int32_t mvy, int32_t satd, int32_t pel, uint32_t *luma,
                      uint32_t *chroma) {
    block_cost_lc(src, ref, level, px, py, bw, bh, mvx, mvy, satd, pel, luma, chroma);
}

/* exact_sad, :1223-1261 */
static u32 exact_sad(const or_planes *src, const or_planes *ref, i32 level, i32 px, i32 py, i32 bw, i32 bh, pt mv,
                     int satd, i32 pel, int include_chroma) {
    if (!include_chroma) {
        pel = imax(pel, 1);
        u32 l, c;
        g_cnt[0]++;
        if (block_cost_edge_lc(src, ref, level, px, py, bw, bh, mv.x, mv.y, satd, pel, &l, &c)) return l;
        return luma_interior(src, ref, level, px, py, i32_as_usize(bw), i32_as_usize(bh), mv.x, mv.y, satd, pel);
    }
    u32 l, c;
    block_cost_lc(src, ref, level, px, py, bw, bh, mv.x, mv.y, satd, pel, &l, &c);
    return sat_add_u32(l, c);
}

static inline i64 motion_penalty(i32 lambda, pt pred, pt mv) { /* :1263-1267 */
    i64 dx = (i64)pred.x - mv.x, dy = (i64)pred.y - mv.y;
    return ((i64)lambda * (dx * dx + dy * dy)) >> 8;
}
static inline int exact_ok(pt mv, bounds_t b) { /* :1275-1277 */
    return mv.x >= b.min_x && mv.y >= b.min_y && mv.x < b.max_x && mv.y < b.max_y;
}
static inline i64 pen(i32 pnew, u32 x) { return (i64)x + (((i64)pnew * (i64)x) >> 8); }

/* exact_sad_if_better, :1158-1221; returns 0 for None */
static int sad_if_better(const or_planes *src, const or_planes *ref, i32 level, i32 px, i32 py, i32 bw, i32 bh,
                         pt mv, int satd, i32 pel, int chroma, i64 motion, i32 pnew, i64 best_cost, u32 *sad_o,
                         i64 *cost_o) {
    pel = imax(pel, 1);
    usize lw, lh;
    level_size(src, level, &lw, &lh);
    i32 t0, t1, t2, t3;
    int shifted = edge_shift_origins(px, py, mv.x, mv.y, bw, bh, (i32)lw, (i32)lh, pel, &t0, &t1, &t2, &t3);
    if (shifted || pnew < 0) {
        u32 luma, colour;
        block_cost_lc(src, ref, level, px, py, bw, bh, mv.x, mv.y, satd, pel, &luma, &colour);
        colour *= (u32)(chroma != 0);
        *sad_o = sat_add_u32(luma, colour);
        *cost_o = motion + pen(pnew, luma) + pen(pnew, colour);
        return 1;
    }
    g_cnt[0]++;
    u32 luma = luma_interior(src, ref, level, px, py, i32_as_usize(bw), i32_as_usize(bh), mv.x, mv.y, satd, pel);
    i64 lower = motion + pen(pnew, luma);
    if (lower >= best_cost) return 0;
    if (!chroma) { *sad_o = luma; *cost_o = lower; return 1; }
    u32 c = chroma_sad_x4(src, ref, level, pel, mv.x, mv.y, i32_as_usize(px), i32_as_usize(py), i32_as_usize(bw),
                          i32_as_usize(bh), lw, lh, satd);
    *sad_o = sat_add_u32(luma, c);
    *cost_o = lower + pen(pnew, c);
    return 1;
}

typedef struct {
    const or_planes *src, *ref;
    i32 level, px, py, bw, bh, pel;
    int satd, chroma;
    pt predictor;
    bounds_t bounds;
    i32 lambda, pnew;
} ctx_t;

/* exact_check, :1122-1155 */
static void exact_check(const ctx_t *c, pt mv, best_t *best) {
    if (!exact_ok(mv, c->bounds)) return;
    i64 motion = motion_penalty(c->lambda, c->predictor, mv);
    if (motion >= best->cost) return;
    u32 sad; i64 cost;
    if (!sad_if_better(c->src, c->ref, c->level, c->px, c->py, c->bw, c->bh, mv, c->satd, c->pel, c->chroma, motion,
                       c->pnew, best->cost, &sad, &cost)) return;
    if (cost < best->cost) { best->mv = mv; best->sad = sad; best->cost = cost; }
}
/* exact_check_dir, :902-939 */
static void exact_check_dir(const ctx_t *c, pt mv, i32 label, i32 *dir, best_t *best) {
    if (!exact_ok(mv, c->bounds)) return;
    i64 motion = motion_penalty(c->lambda, c->predictor, mv);
    if (motion >= best->cost) return;
    u32 sad; i64 cost;
    if (!sad_if_better(c->src, c->ref, c->level, c->px, c->py, c->bw, c->bh, mv, c->satd, c->pel, c->chroma, motion,
                       c->pnew, best->cost, &sad, &cost)) return;
    if (cost < best->cost) { best->sad = sad; best->cost = cost; *dir = label; }
}
/* exact_expanding, :829-886 */
static void exact_expanding(const ctx_t *c, pt center, i32 radius, i32 step, best_t *best) {
    for (i32 i = -radius + step; i < radius; i += step) {
        exact_check(c, (pt){center.x + i, center.y - radius}, best);
        exact_check(c, (pt){center.x + i, center.y + radius}, best);
    }
    for (i32 j = -radius + step; j < radius; j += step) {
        exact_check(c, (pt){center.x - radius, center.y + j}, best);
        exact_check(c, (pt){center.x + radius, center.y + j}, best);
    }
    exact_check(c, (pt){center.x - radius, center.y - radius}, best);
    exact_check(c, (pt){center.x - radius, center.y + radius}, best);
    exact_check(c, (pt){center.x + radius, center.y - radius}, best);
    exact_check(c, (pt){center.x + radius, center.y + radius}, best);
}

static const pt HEX2[8] = {{-1, -2}, {-2, 0}, {-1, 2}, {1, 2}, {2, 0}, {1, -2}, {-1, -2}, {-2, 0}}; /* :889-898 */
static const i32 MOD6M1[8] = {5, 0, 1, 2, 3, 4, 5, 0};

/* exact_hex2, :942-1033 */
static void exact_hex2(const ctx_t *c, i32 radius, best_t *best) {
    i32 bmx = best->mv.x, bmy = best->mv.y;
    if (radius > 1) {
        i32 dir = -2;
        for (i32 i = 0; i < 6; i++) exact_check_dir(c, (pt){bmx + HEX2[i + 1].x, bmy + HEX2[i + 1].y}, i, &dir, best);
        if (dir != -2) {
            bmx += HEX2[dir + 1].x; bmy += HEX2[dir + 1].y;
            i32 i = 1;
            while (i < radius / 2 && exact_ok((pt){bmx, bmy}, c->bounds)) {
                i32 odir = MOD6M1[dir + 1];
                dir = -2;
                for (i32 k = 0; k < 3; k++)
                    exact_check_dir(c, (pt){bmx + HEX2[odir + k].x, bmy + HEX2[odir + k].y}, odir + k - 1, &dir, best);
                if (dir == -2) break;
                bmx += HEX2[dir + 1].x; bmy += HEX2[dir + 1].y;
                i += 1;
            }
        }
        best->mv = (pt){bmx, bmy};
    }
    exact_expanding(c, (pt){bmx, bmy}, 1, 1, best);
}

static const pt HEX4[16] = {{-4, 2}, {-4, 1}, {-4, 0}, {-4, -1}, {-4, -2}, {4, -2}, {4, -1}, {4, 0},
                            {4, 1},  {4, 2},  {2, 3},  {0, 4},   {-2, 3},  {-2, -3}, {0, -4}, {2, -3}};
/* exact_umh, :1036-1119 */
static void exact_umh(const ctx_t *c, pt center, i32 radius, best_t *best) {
    for (i32 d = 1; d < radius; d += 2) {
        exact_check(c, (pt){center.x - d, center.y}, best);
        exact_check(c, (pt){center.x + d, center.y}, best);
    }
    for (i32 d = 1; d < radius; d += 2) {
        exact_check(c, (pt){center.x, center.y - d}, best);
        exact_check(c, (pt){center.x, center.y + d}, best);
    }
    i32 smax = imax(radius / 4, 1);
    for (i32 s = 1; s <= smax; s++)
        for (int k = 0; k < 16; k++) exact_check(c, (pt){center.x + HEX4[k].x * s, center.y + HEX4[k].y * s}, best);
    exact_hex2(c, radius, best);
}

/* exact_refine_search, :771-826 */
static void exact_refine_search(const ctx_t *c, i32 search_type, i32 radius, best_t *best) {
    if (search_type == 2) exact_hex2(c, radius, best);
    else if (search_type == 3) exact_umh(c, best->mv, radius, best);
    else if (search_type == 4) {
        i32 cx = best->mv.x, cy = best->mv.y;
        for (i32 y = cy - radius; y <= cy + radius; y++)
            for (i32 x = cx - radius; x <= cx + radius; x++) exact_check(c, (pt){x, y}, best);
    }
}

/* exact_search_block, :684-768 */
static best_t exact_search_block(ctx_t *c, const or_analyse_opts *o, int field_valid, const or_vec8 *prev, pt zero,
                                 pt global, const pt *nb, int nnb, i32 search_type, i32 radius) {
#define SPECIAL(mv_, pen_, out_)                                                                                \
    do {                                                                                                        \
        u32 s_ = exact_sad(c->src, c->ref, c->level, c->px, c->py, c->bw, c->bh, (mv_), c->satd, c->pel,        \
                           c->chroma);                                                                          \
        (out_).mv = (mv_); (out_).sad = s_; (out_).cost = (i64)s_ + (((i64)(pen_) * (i64)s_) >> 8);             \
    } while (0)
    best_t field = {{0, 0}, 0, 0}, previous, zero_b, global_b;
    if (field_valid) SPECIAL(c->predictor, 0, field);
    if (c->level == 0 && o->distance == 0) {
        if (field_valid) return field;
        best_t z;
        SPECIAL(zero, 0, z);
        return z;
    }
    if (prev) SPECIAL(((pt){prev->dx, prev->dy}), o->prev, previous);
    SPECIAL(zero, o->pzero, zero_b);
    SPECIAL(global, o->pglobal, global_b);
    best_t best;
    if (field_valid) best = field;
    else { best.mv = zero; best.sad = UINT32_MAX; best.cost = INT64_MAX; }
    if (prev && previous.cost < best.cost) { best = previous; c->predictor = previous.mv; }
    if (global_b.cost < best.cost) best = global_b;
    if (zero_b.cost < best.cost) best = zero_b;
    for (int k = 0; k < nnb; k++) {
        u32 sad = exact_sad(c->src, c->ref, c->level, c->px, c->py, c->bw, c->bh, nb[k], c->satd, c->pel, c->chroma);
        i64 cost = (i64)sad + (((i64)o->pnbour * (i64)sad) >> 8);
        if (cost < best.cost) { best.mv = nb[k]; best.sad = sad; best.cost = cost; }
    }
    best.cost = (i64)best.sad;
    exact_refine_search(c, search_type, radius, &best);
    return best;
#undef SPECIAL
}

static i32 search_radius(const or_analyse_opts *o, int fine, i32 level, i32 nlevels) { /* :1465-1476 */
    i32 d = fine ? o->distance : o->coarse_distance;
    if (d == 0) return (level == 0 && nlevels > 1) ? 0 : 10;
    return iabs(d);
}
static i32 adaptive_radius(i32 radius, u32 activity) { /* :1478-1484 */
    if (activity < 2) return 0;
    u32 a = 255u * activity / 150u;
    return ((radius * (i32)(a < 255 ? a : 255)) >> 8) + 1;
}
static u32 plane_activity(const px *data, usize len, usize stride, usize row, usize x, usize width, usize height,
                          int satd) { /* :1517-1553 */
    u32 area = (u32)(width * height);
    u32 sum = 0;
    for (usize y = 0; y < height; y++)
        for (usize c = 0; c < width; c++) sum += read_or(data, len, (row + y) * stride + x + c, 0);
    u32 mean = sum / area;
    if (!satd) {
        u32 s = 0;
        for (usize y = 0; y < height; y++)
            for (usize c = 0; c < width; c++) {
                u32 v = read_or(data, len, (row + y) * stride + x + c, 0);
                s += v > mean ? v - mean : mean - v;
            }
        return s / area;
    }
    u32 total = 0;
    for (usize y = 0; y < height; y += 4)
        for (usize x0 = 0; x0 < width; x0 += 4) {
            i32 d[16];
            for (usize dy = 0; dy < 4; dy++)
                for (usize dx = 0; dx < 4; dx++)
                    d[dy * 4 + dx] = (i32)read_or(data, len, (row + y + dy) * stride + x + x0 + dx, 0) - (i32)mean;
            total += or_hadamard4_satd(d);
        }
    return (total >> 1) / area;
}
static u32 block_activity(const or_planes *src, i32 level, i32 px, i32 py, i32 bw, i32 bh, int satd) { /* :1486-1515 */
    usize lw, lh;
    level_size(src, level, &lw, &lh);
    i32 x = px - (level > 0 && px + bw >= (i32)lw), y = py - (level > 0 && py + bh >= (i32)lh);
    u32 luma = plane_activity(src->y, src->y_len, src->y_stride, level_y_offset(src, level) + i32_as_usize(y),
                              i32_as_usize(x), i32_as_usize(bw), i32_as_usize(bh), satd);
    usize cw = i32_as_usize(bw / 2), ch = i32_as_usize(bh / 2);
    usize off = chroma_level_offset(src, level);
    return luma +
           plane_activity(src->u, src->u_len, src->u_stride, off + i32_as_usize(py / 2), i32_as_usize(px / 2), cw, ch, satd) +
           plane_activity(src->v, src->v_len, src->v_stride, off + i32_as_usize(py / 2), i32_as_usize(px / 2), cw, ch, satd);
}

int32_t or_adapt_lambda(int32_t nlambda, int32_t lsad, uint32_t pred_score) { /* :1555-1564 */
    double l = (double)imax(lsad, 1);
    double half_score = pred_score == UINT32_MAX ? -1.0 : (double)(pred_score >> 1);
    double t = l / (l + half_score);
    return f64_as_i32(fmin((double)nlambda * t * t, 21474836.47));
}
static double powi_(double a, i32 b) { /* llvm.powi lowering (compiler-rt __powidf2) */
    int recip = b < 0;
    double r = 1;
    for (;;) {
        if (b & 1) r *= a;
        b /= 2;
        if (b == 0) break;
        a *= a;
    }
    return recip ? 1 / r : r;
}
int32_t or_exact_lambda(const or_analyse_opts *o, int32_t level, int32_t pel) { /* :1279-1283 */
    return f64_as_i32((double)o->lambda / powi_(o->plevel, o->levels - level - 1) / (double)imax(pel * pel, 1));
}

static u8 block_luma_dc(const or_planes *src, i32 level, i32 px, i32 py, i32 bw, i32 bh) { /* :1566-1617 */
    usize lw, lh;
    level_size(src, level, &lw, &lh);
    usize y_off = level_y_offset(src, level);
    if (is_blk(i32_as_usize(bw)) && is_blk(i32_as_usize(bh)) && px >= 0 && py >= 0 && (usize)px + (usize)bw <= lw &&
        (usize)py + (usize)bh <= lh) {
        usize w = (usize)bw, h = (usize)bh;
        usize start = (y_off + (usize)py) * src->y_stride + (usize)px;
        usize end = sat_add_us(start, (h - 1) * src->y_stride + w);
        if (end <= src->y_len) {
            u32 sum = 0;
            for (usize r = 0; r < h; r++)
                for (usize c = 0; c < w; c++) sum += src->y[start + r * src->y_stride + c];
            u32 m = sum / (u32)(w * h);
            m >>= DC_SHIFT;
            return (u8)(m < 255 ? m : 255);
        }
    }
    u32 sum = 0, count = 0;
    for (usize row = 0; row < i32_as_usize(bh); row++) {
        usize y = i32_as_usize(py) + row;
        if (y >= lh) break;
        for (usize col = 0; col < i32_as_usize(bw); col++) {
            usize x = i32_as_usize(px) + col;
            if (x >= lw) break;
            sum += read_or(src->y, src->y_len, (y_off + y) * src->y_stride + x, 0);
            count++;
        }
    }
    if (count == 0) return 0;
    u32 m = sum / count;
    m >>= DC_SHIFT;
    return (u8)(m < 255 ? m : 255);
}

static int cmp_i32(const void *a, const void *b) {
    i32 x = *(const i32 *)a, y = *(const i32 *)b;
    return (x > y) - (x < y);
}
void or_global_doubled(const or_vec8 *field, size_t n, int32_t *gx, int32_t *gy) { /* :1285-1324 */
    i32 *vals = malloc((n ? n : 1) * sizeof(i32));
    i32 m[2];
    for (int comp = 0; comp < 2; comp++) {
        for (usize i = 0; i < n; i++) vals[i] = comp == 0 ? field[i].dx : field[i].dy;
        qsort(vals, n, sizeof(i32), cmp_i32);
        i32 best = n ? vals[0] : 0;
        usize best_count = 0, i = 0;
        while (i < n) {
            i32 value = vals[i];
            usize j = i + 1;
            while (j < n && vals[j] == value) j++;
            if (j - i > best_count) { best = value; best_count = j - i; }
            i = j;
        }
        m[comp] = best;
    }
    free(vals);
    i64 sx = 0, sy = 0, count = 0;
    for (usize i = 0; i < n; i++) {
        if (iabs((i32)field[i].dx - m[0]) < 6 && iabs((i32)field[i].dy - m[1]) < 6) {
            sx += field[i].dx; sy += field[i].dy; count++;
        }
    }
    if (count == 0) { *gx = 2 * m[0]; *gy = 2 * m[1]; return; }
    i64 ssx = (sx > 0) - (sx < 0), ssy = (sy > 0) - (sy < 0);
    *gx = 2 * (i32)((sx + ssx * count / 2) / count);
    *gy = 2 * (i32)((sy + ssy * count / 2) / count);
}

/* ---- search orders, :302-419 */
typedef struct { pt *v; usize n, cap; } ptvec;
static void pv_push(ptvec *a, i32 x, i32 y) {
    if (a->n == a->cap) { a->cap = a->cap ? 2 * a->cap : 64; a->v = realloc(a->v, a->cap * sizeof(pt)); }
    a->v[a->n++] = (pt){x, y};
}
static void initial_search_order(ptvec *o, i32 gw, i32 gh) { /* :302-324 */
    for (i32 y = 1; y < gh - 1; y++) {
        if ((y & 1) == 0) for (i32 x = 1; x < gw - 1; x++) pv_push(o, x, y);
        else for (i32 x = gw - 2; x >= 1; x--) pv_push(o, x, y);
    }
    for (i32 x = 0; x < gw; x++) { pv_push(o, x, 0); if (gh > 1) pv_push(o, x, gh - 1); }
    for (i32 y = 1; y < gh - 1; y++) { pv_push(o, 0, y); if (gw > 1) pv_push(o, gw - 1, y); }
}
static void level_search_order(ptvec *o, i32 gw, i32 gh, i32 level) { /* :326-336 */
    i32 edge = level > 0, bw = gw - edge, bh = gh - edge;
    o->n = 0;
    initial_search_order(o, bw, bh);
    if (edge) {
        for (i32 x = 0; x <= bw; x++) pv_push(o, x, bh);
        for (i32 y = 0; y < bh; y++) pv_push(o, bw, y);
    }
}
static void refine_search_order(ptvec *out, const ptvec *coarse, i32 cgw, i32 cgh, i32 gw, i32 gh, i32 level) {
    out->n = 0; /* :338-402 */
    if (level == 0) { initial_search_order(out, gw, gh); return; }
    i32 sw = cgw - 1, sh = cgh - 1, dw = gw - 1, dh = gh - 1;
    i32 extra_x = imax(dw - 2 * sw, 0), extra_y = imax(dh - 2 * sh, 0);
    ptvec boundary = {0};
    usize ns = (usize)imax(gw * gh, 0);
    u8 *seen = calloc(ns ? ns : 1, 1);
#define ADD(cx_, cy_)                                                                                           \
    do {                                                                                                        \
        i32 x_ = (cx_), y_ = (cy_);                                                                             \
        if (!(x_ < 0 || y_ < 0 || x_ >= dw || y_ >= dh)) {                                                      \
            usize ix_ = (usize)(y_ * gw + x_);                                                                  \
            if (!seen[ix_]) {                                                                                   \
                seen[ix_] = 1;                                                                                  \
                if (x_ > 0 && y_ > 0 && x_ < dw - 1 && y_ < dh - 1) pv_push(out, x_, y_);                       \
                else pv_push(&boundary, x_, y_);                                                                \
            }                                                                                                   \
        }                                                                                                       \
    } while (0)
    for (usize k = 0; k < coarse->n; k++) {
        i32 x = coarse->v[k].x, y = coarse->v[k].y;
        if (x >= sw || y >= sh) continue;
        i32 left = 2 * x, top = 2 * y;
        ADD(left, top); ADD(left + 1, top); ADD(left + 1, top + 1); ADD(left, top + 1);
        if (x == sw - 1)
            for (i32 dx = 2; dx < 2 + extra_x; dx++)
                for (i32 dy = 0; dy < 2 + (y == sh - 1) * extra_y; dy++) ADD(left + dx, top + dy);
        if (y == sh - 1)
            for (i32 dy = 2; dy < 2 + extra_y; dy++)
                for (i32 dx = 0; dx < 2; dx++) ADD(left + dx, top + dy);
    }
#undef ADD
    for (usize k = 0; k < boundary.n; k++) pv_push(out, boundary.v[k].x, boundary.v[k].y);
    for (i32 x = 0; x <= dw; x++) pv_push(out, x, dh);
    for (i32 y = 0; y < dh; y++) pv_push(out, dw, y);
    free(boundary.v);
    free(seen);
}
typedef struct { u32 key; u32 idx; } skey;
static int cmp_skey(const void *a, const void *b) { /* stable: (key, original index) */
    const skey *x = a, *y = b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return (x->idx > y->idx) - (x->idx < y->idx);
}
static void reorder_search_order(ptvec *order, const or_vec8 *field, i32 gw, i32 gh, i32 bw, i32 bh) { /* :404-419 */
    usize count = (usize)((gw - 1) * (gh - 1));
    u32 v = (u32)imax(bw * bh / 8, 1), lg = 0;
    while (v >>= 1) lg++;
    u32 shift = lg + 1;
    skey *k = malloc((count ? count : 1) * sizeof(skey));
    usize n = 0;
    for (i32 y = 0; y < gh - 1; y++)
        for (i32 x = 0; x < gw - 1; x++) { k[n].key = field[y * gw + x].score >> shift; k[n].idx = (u32)n; n++; }
    qsort(k, n, sizeof(skey), cmp_skey);
    for (usize i = 0; i < n; i++) {
        u32 id = k[i].idx;
        order->v[i] = (pt){(i32)(id % (u32)(gw - 1)), (i32)(id / (u32)(gw - 1))};
    }
    free(k);
}

/* exact_interpolate_level, :421-478 */
static void interpolate_level(const or_vec8 *coarse, i32 cgw, i32 cgh, i32 gw, i32 gh, i32 bw, i32 bh, i32 ox, i32 oy,
                              i32 pel, or_vec8 *out, or_vec8 *projected) {
    usize n = (usize)(gw * gh);
    memset(out, 0, n * sizeof(or_vec8));
    for (usize i = 0; i < n; i++) { memset(&projected[i], 0, sizeof(or_vec8)); projected[i].score = UINT32_MAX; }
    i32 cw = cgw - 1, ch = cgh - 1;
    for (i32 y = 0; y < gh - 1; y++)
        for (i32 x = 0; x < gw - 1; x++) {
            or_vec8 p;
            if (x < 2 * cw && y < 2 * ch) p = coarse[(y >> 1) * cgw + (x >> 1)];
            else {
                i32 edge = ch + imin(x >> 1, cw) - imin(y >> 1, ch);
                i32 ex, ey;
                if (edge <= cw) { ex = edge; ey = ch; } else { ex = cw; ey = cw + ch - edge; }
                p = coarse[ey * cgw + ex];
            }
            i32 vx = (i32)p.dx * 2 * pel, vy = (i32)p.dy * 2 * pel;
            or_vec8 vec = p;
            vec.dx = (int16_t)iclamp(vx, -32768, 32767);
            vec.dy = (int16_t)iclamp(vy, -32768, 32767);
            out[y * gw + x] = vec;
            if (x >= 2 * cw || y >= 2 * ch) continue;
            i32 tx = iclamp((vx + (bw >> 1) + (bw - ox) * x) / (bw - ox), 0, gw - 1);
            i32 ty = iclamp((vy + (bh >> 1) + (bh - oy) * y) / (bh - oy), 0, gh - 1);
            or_vec8 *t = &projected[ty * gw + tx];
            if (vec.score < t->score) {
                memset(t, 0, sizeof(*t));
                t->dx = (int16_t)-vec.dx; t->dy = (int16_t)-vec.dy; t->score = vec.score; t->luma = 0;
            }
        }
}

/* exact_search_level, :480-681; returns 0, or -1 where the reference would panic */
static int search_level(const or_planes *src, const or_planes *ref, const or_analyse_opts *o, i32 level, pt global,
                        const or_vec8 *prev, usize prev_len, or_vec8 *field, i32 gw, i32 gh, const ptvec *order) {
    i32 bw0 = o->block_w, bh0 = o->block_h;
    i32 step_x = imax(bw0 - o->overlap_x, 1), step_y = imax(bh0 - o->overlap_y, 1);
    i32 pel = level == 0 ? imax(o->pel, 1) : 1;
    i32 base_radius = search_radius(o, level == 0, level, imax(o->levels, 1));
    i32 search_type = level == 0 ? o->search_type : o->coarse_search_type;
    int satd = level == 0 ? o->fine_satd : o->coarse_satd;
    i32 bad_count = 0;
    usize nfield = (usize)(gw * gh);
    usize psz = (usize)imax((gw + 1) * (gh + 1), 0);
    u8 *processed = calloc(psz ? psz : 1, 1);
    usize lw_, lh_;
    level_size(src, level, &lw_, &lh_);
    i32 lw = (i32)lw_, lh = (i32)lh_;
    for (usize k = 0; k < order->n; k++) {
        i32 bx = order->v[k].x, by = order->v[k].y;
        usize idx = i32_as_usize(by * gw + bx);
        i32 px = (level > 0 && bx == gw - 1) ? lw - bw0 : bx * step_x;
        i32 py = (level > 0 && by == gh - 1) ? lh - bh0 : by * step_y;
        int smallest = level == o->levels - 1;
        i32 bw = bw0, bh = bh0;
        if (smallest) { px += bw0 >> 2; py += bh0 >> 2; bw = bw0 >> 1; bh = bh0 >> 1; }
        bounds_t bounds = mv_bounds(px, py, bw, bh, lw, lh, pel);
        int edge = level > 0 && (bx == gw - 1 || by == gh - 1);
        i32 sx = imin(bx, gw - 2), sy = imin(by, gh - 2);
        usize sidx = i32_as_usize(sy * gw + sx);
        if (sidx >= nfield || idx >= nfield) { free(processed); return -1; }
        or_vec8 interp = field[sidx];
        if (edge && !smallest)
            interp.score = exact_sad(src, ref, level, sx * step_x, sy * step_y, bw, bh, (pt){interp.dx, interp.dy},
                                     satd, pel, 1);
        else if (!edge) interp = field[idx];
        or_vec8 predictor = interp;
        pt pred_mv = {predictor.dx, predictor.dy};
        i32 lambda_base = smallest ? 0 : or_exact_lambda(o, level, pel);
        i32 lambda = or_adapt_lambda(lambda_base, smallest ? o->lsad / 3 : o->lsad, predictor.score);
        i32 radius = base_radius;
        if (level > 0 && o->coarse_distance < 0)
            radius = adaptive_radius(base_radius, block_activity(src, level, px, py, bw, bh, satd));
        pt seeds[9];
        int ns = 0;
        for (i32 ny = imax(by - 1, 0); ny <= imin(by + 1, gh - 1); ny++)
            for (i32 nx = imax(bx - 1, 0); nx <= imin(bx + 1, gw - 1); nx++)
                if (processed[ny * (gw + 1) + nx]) {
                    if (ns >= 8) { free(processed); return -1; } /* seeds[8] overflow panics */
                    seeds[ns++] = (pt){field[ny * gw + nx].dx, field[ny * gw + nx].dy};
                }
        const or_vec8 *pv = NULL;
        if (idx < prev_len && prev[idx].score != UINT32_MAX && prev[idx].score > 0) pv = &prev[idx];
        ctx_t c = {src, ref, level, px, py, bw, bh, pel, satd, !smallest, pred_mv, bounds, lambda, o->pnew};
        best_t best = exact_search_block(&c, o, predictor.score != UINT32_MAX, pv, (pt){0, 0}, global, seeds, ns,
                                         (edge && level == 1) ? 0 : search_type, radius);
        u32 found = best.sad;
        i32 bad_limit = sat_add_i32(o->coarse_bad_sad, sat_mul_i32(o->coarse_bad_sad, bad_count) / 16);
        if (level < 16) g_lvl[level][1] = g_cnt[0];
        if (level > 0 && idx > 1 && o->coarse_bad_sad > 0 && (i32)best.sad > bad_limit) {
            bad_count += 1;
            u64 e0 = g_cnt[0];
            if (level < 16) g_lvl[level][2]++;
            ctx_t e = c; /* pred_mv of the block, not a re-anchored one */
            e.predictor = pred_mv;
            if (o->coarse_bad_range < 0) {
                i32 max_r = -o->coarse_bad_range * pel;
                for (i32 r = pel; r < max_r; r += pel) {
                    exact_expanding(&e, (pt){0, 0}, r, pel, &best);
                    if (best.sad < found / 4) break;
                }
            } else if (o->coarse_bad_range > 0) {
                exact_umh(&e, (pt){0, 0}, o->coarse_bad_range * pel, &best);
            }
            pt center = best.mv;
            exact_expanding(&e, center, 1, 1, &best);
            if (level < 16) g_lvl[level][3] += g_cnt[0] - e0;
        }
        if (level < 16) { g_lvl[level][0]++; }
        field[idx].dx = (int16_t)best.mv.x;
        field[idx].dy = (int16_t)best.mv.y;
        field[idx].score = sat_mul_u32(best.sad, smallest ? 3 : 1);
        field[idx].luma = block_luma_dc(src, level, px, py, bw, bh);
        processed[by * (gw + 1) + bx] = 1;
    }
    free(processed);
    return 0;
}

/* exact_recalculate, :1326-1451 */
static i64 div_euclid(i64 a, i64 b) {
    i64 q = a / b, r = a % b;
    if (r < 0) q = b > 0 ? q - 1 : q + 1;
    return q;
}
static void exact_clip(pt *mv, bounds_t b) { /* :1269-1273 */
    i32 max_x = imax(b.max_x - 1, b.min_x), max_y = imax(b.max_y - 1, b.min_y);
    mv->x = iclamp(mv->x, b.min_x, max_x);
    mv->y = iclamp(mv->y, b.min_y, max_y);
}
static or_vec8 *recalculate(const or_planes *src, const or_planes *ref, const or_analyse_opts *o, or_vec8 *field,
                            i32 old_gw, i32 old_gh, i32 *ogw, i32 *ogh) {
    if (!o->has_refine_thsad) { *ogw = old_gw; *ogh = old_gh; return field; }
    i32 thsad = o->refine_thsad;
    i32 old_bw = o->block_w, old_bh = o->block_h, old_ox = o->overlap_x, old_oy = o->overlap_y;
    i32 bw, bh, ox, oy, gw, gh;
    or_output_block(o, &bw, &bh, &ox, &oy);
    or_grid(o, bw, bh, ox, oy, &gw, &gh);
    i32 osx = imax(old_bw - old_ox, 1), osy = imax(old_bh - old_oy, 1);
    i32 step_x = imax(bw - ox, 1), step_y = imax(bh - oy, 1);
    i32 pel = imax(o->pel, 1);
    usize lw, lh;
    level_size(src, 0, &lw, &lh);
    or_vec8 *out = calloc((usize)(gw * gh), sizeof(or_vec8));
    for (i32 by = 0; by < gh; by++)
        for (i32 bx = 0; bx < gw; bx++) {
            i32 center_x = bw / 2 + step_x * bx, center_y = bh / 2 + step_y * by;
            i32 old_x = (center_x - old_bw / 2) / osx, old_y = (center_y - old_bh / 2) / osy;
            i32 delta_x = imax(center_x - (old_bw / 2 + osx * old_x), 0);
            i32 delta_y = imax(center_y - (old_bh / 2 + osy * old_y), 0);
#define GET(x_, y_) field[iclamp((y_), 0, old_gh - 1) * old_gw + iclamp((x_), 0, old_gw - 1)]
            or_vec8 p00 = GET(old_x, old_y), p10 = GET(old_x + 1, old_y), p01 = GET(old_x, old_y + 1),
                    p11 = GET(old_x + 1, old_y + 1);
#undef GET
#define INTERP(a_, b_, c_, d_)                                                                                  \
    div_euclid(((i64)(a_) * osx + (i64)delta_x * ((i64)(b_) - (a_))) +                                          \
                   div_euclid((i64)delta_y * (((i64)(c_) * osx + (i64)delta_x * ((i64)(d_) - (c_))) -           \
                                              ((i64)(a_) * osx + (i64)delta_x * ((i64)(b_) - (a_)))),           \
                              (i64)osy),                                                                        \
               (i64)osx)
            pt mv = {(i32)INTERP(p00.dx, p10.dx, p01.dx, p11.dx), (i32)INTERP(p00.dy, p10.dy, p01.dy, p11.dy)};
            i64 parent_sad = INTERP((i64)p00.score, (i64)p10.score, (i64)p01.score, (i64)p11.score) *
                             (i64)(bw * bh) / (i64)(old_bw * old_bh);
#undef INTERP
            i32 px = bx * step_x, py = by * step_y;
            int border = bx == 0 || by == 0 || bx == gw - 1 || by == gh - 1;
            i32 factor = (border && bw > 4) ? 3 : 1;
            i32 ebw = factor == 3 ? bw / 2 : bw, ebh = factor == 3 ? bh / 2 : bh;
            i32 epx = px + (factor == 3 ? bw / 4 : 0), epy = py + (factor == 3 ? bh / 4 : 0);
            bounds_t bounds = mv_bounds(epx, epy, ebw, ebh, (i32)lw, (i32)lh, pel);
            pt predictor = mv;
            exact_clip(&predictor, bounds);
            i64 ps0 = lmax(parent_sad, 0);
            best_t best = {predictor, (u32)(ps0 < (i64)UINT32_MAX ? ps0 : (i64)UINT32_MAX), ps0};
            i32 threshold = thsad / factor;
            if (parent_sad > (i64)threshold) {
                best.sad = exact_sad(src, ref, 0, epx, epy, ebw, ebh, predictor, o->refine_satd, pel, 1);
                best.cost = (i64)best.sad;
                i32 lambda = by == 0 ? 0 : (o->lambda >> 2) / factor;
                ctx_t c = {src, ref, 0, epx, epy, ebw, ebh, pel, o->refine_satd, 1, predictor, bounds, lambda,
                           o->pnew / factor};
                exact_refine_search(&c, o->refine_search_type, iabs(o->refine_distance), &best);
            }
            or_vec8 *v = &out[by * gw + bx];
            v->dx = (int16_t)best.mv.x; v->dy = (int16_t)best.mv.y;
            v->score = sat_mul_u32(best.sad, (u32)factor);
            v->luma = block_luma_dc(src, 0, epx, epy, ebw, ebh);
        }
    free(field);
    *ogw = gw; *ogh = gh;
    return out;
}

void or_rescale_scores(or_vec8 *field, size_t n, int32_t width, int32_t height, int32_t blk) { /* :2716-2738 */
    double f = sqrt(powi_((double)width, 2) + powi_((double)height, 2));
    i32 diag = imax(f64_as_i32(f), 0);
    i32 denom = imax(sat_mul_i32(diag, imax(blk, 1)), 1);
    for (usize i = 0; i < n; i++) {
        or_vec8 *v = &field[i];
        i32 mag = iabs(v->dx) + iabs(v->dy);
        i32 ratio = (100 * mag) / denom;
        i32 score = (i32)v->score;
        if (ratio >= 51) score = sat_mul_i32(score, 20);
        else if (ratio >= 16) {
            u64 v71 = ((u64)3926827243u * (u64)(u32)score * (u64)(u32)(ratio - 15)) >> 32;
            i32 w = (i32)(u32)v71;
            score = sat_add_i32(score, 9 * ((w >> 31) + (w >> 5)));
        }
        v->score = (u32)score & 0x00FFFFFFu;
    }
}

/* exact_search_hierarchy{,_bidir}, :94-293. dirs: bit0 = bwd, bit1 = fwd. */
typedef struct {
    or_vec8 *field, *next, *prev_proj;
    ptvec order;
    pt global;
} dir_state;

int or_analyse_pair(const or_planes *cur, const or_planes *ref, const or_analyse_opts *o, or_vec8 *bwd_out,
                    or_vec8 *fwd_out) {
    memset(g_cnt, 0, sizeof(g_cnt));
    memset(g_lvl, 0, sizeof(g_lvl));
    int do_bwd = (o->vectors & 1) != 0, do_fwd = (o->vectors & 2) != 0;
    /* In the bidir form fwd searches cur->ref and bwd searches ref->cur with the other
     * direction's projection as `prev`; single-direction forms pass an empty prev. */
    int bidir = do_bwd && do_fwd;
    dir_state st[2];
    memset(st, 0, sizeof(st)); /* 0 = fwd (cur, ref), 1 = bwd (ref, cur) */
    i32 field_gw = 0, field_gh = 0;
    int rc = 0;
    int active[2] = {do_fwd, do_bwd};
    for (i32 level = imax(o->levels, 1) - 1; level >= 0 && rc == 0; level--) {
        i32 gw, gh;
        or_level_grid(o, level, &gw, &gh);
        i32 pel = level == 0 ? imax(o->pel, 1) : 1;
        usize n = (usize)(gw * gh);
        for (int d = 0; d < 2; d++) {
            if (!active[d]) continue;
            dir_state *s = &st[d];
            if (s->order.n == 0) level_search_order(&s->order, gw, gh, level);
            else {
                ptvec t = {0};
                refine_search_order(&t, &s->order, field_gw, field_gh, gw, gh, level);
                free(s->order.v);
                s->order = t;
            }
            s->next = malloc(n * sizeof(or_vec8));
            if (!s->field) {
                memset(s->next, 0, n * sizeof(or_vec8));
                free(s->prev_proj);
                s->prev_proj = NULL;
            } else {
                free(s->prev_proj);
                s->prev_proj = malloc(n * sizeof(or_vec8));
                interpolate_level(s->field, field_gw, field_gh, gw, gh, o->block_w, o->block_h, o->overlap_x,
                                  o->overlap_y, pel, s->next, s->prev_proj);
            }
        }
        for (int d = 0; d < 2 && rc == 0; d++) {
            if (!active[d]) continue;
            const or_planes *a = d == 0 ? cur : ref, *b = d == 0 ? ref : cur;
            const or_vec8 *pp = NULL;
            usize plen = 0;
            if (bidir) { pp = st[1 - d].prev_proj; plen = pp ? n : 0; }
            else { pp = st[d].prev_proj; plen = pp ? n : 0; }
            rc = search_level(a, b, o, level, st[d].global, pp, plen, st[d].next, gw, gh, &st[d].order);
        }
        for (int d = 0; d < 2; d++) {
            if (!active[d]) continue;
            dir_state *s = &st[d];
            if (level > 0) {
                or_global_doubled(s->next, n, &s->global.x, &s->global.y);
                reorder_search_order(&s->order, s->next, gw, gh, o->block_w, o->block_h);
            }
            free(s->field);
            s->field = s->next;
            s->next = NULL;
        }
        field_gw = gw; field_gh = gh;
    }
    i32 bw, bh, ox, oy;
    or_output_block(o, &bw, &bh, &ox, &oy);
    for (int d = 0; d < 2; d++) {
        if (!active[d]) continue;
        const or_planes *a = d == 0 ? cur : ref, *b = d == 0 ? ref : cur;
        if (rc == 0) {
            i32 ogw, ogh;
            st[d].field = recalculate(a, b, o, st[d].field, field_gw, field_gh, &ogw, &ogh);
            usize n = (usize)(ogw * ogh);
            or_rescale_scores(st[d].field, n, o->width, o->height, bw);
            or_vec8 *dst = d == 0 ? fwd_out : bwd_out;
            if (dst) memcpy(dst, st[d].field, n * sizeof(or_vec8));
        }
        free(st[d].field);
        free(st[d].prev_proj);
        free(st[d].order.v);
        free(st[d].next);
    }
    for (int i = 0; i < 5; i++) __atomic_fetch_add(&g_tot[i], g_cnt[i], __ATOMIC_RELAXED);
    return rc;
}

size_t or_payload_len(const or_analyse_opts *o) {
    i32 bw, bh, ox, oy, gw, gh;
    or_output_block(o, &bw, &bh, &ox, &oy);
    or_grid(o, bw, bh, ox, oy, &gw, &gh);
    usize nreg = (o->vectors == 1 || o->vectors == 2) ? 1 : 2;
    return 0x40 + nreg * (4 + (usize)(gw * gh) * 8);
}

static void wr32(u8 *b, usize off, u32 v) { b[off] = (u8)v; b[off + 1] = (u8)(v >> 8); b[off + 2] = (u8)(v >> 16); b[off + 3] = (u8)(v >> 24); }

void or_pack_vector_frame(const or_analyse_opts *o, const or_vec8 *previous, const or_vec8 *current, uint8_t *out) {
    i32 bw, bh, ox, oy, gw, gh; /* pack_vector_frame, :2740-2811 */
    or_output_block(o, &bw, &bh, &ox, &oy);
    or_grid(o, bw, bh, ox, oy, &gw, &gh);
    usize count = (usize)(gw * gh);
    i32 flags = (previous ? 1 : 0) | (current ? 2 : 0);
    usize nreg = (previous ? 1 : 0) + (current ? 1 : 0);
    usize total = 0x40 + nreg * (4 + count * 8);
    memset(out, 0, total);
    wr32(out, 0, 16); wr32(out, 4, 0xA0); wr32(out, 8, (u32)flags); wr32(out, 0x0C, (u32)bw);
    wr32(out, 0x10, (u32)bh); wr32(out, 0x14, (u32)o->pel);
    wr32(out, 0x18, (u32)(o->has_refine_thsad ? 1 : o->levels)); wr32(out, 0x1C, 0);
    wr32(out, 0x20, (u32)o->width); wr32(out, 0x24, (u32)o->height); wr32(out, 0x28, (u32)ox);
    wr32(out, 0x2C, (u32)oy); wr32(out, 0x30, (u32)gw); wr32(out, 0x34, (u32)gh);
    wr32(out, 0x38, (u32)o->selector); wr32(out, 0x3C, (u32)o->delta);
    usize cursor = 0x40;
    u32 marker = (u32)(2 * count + 1);
    const or_vec8 *regs[2] = {previous, current};
    for (int r = 0; r < 2; r++) {
        if (!regs[r]) continue;
        wr32(out, cursor, marker);
        cursor += 4;
        for (usize i = 0; i < count; i++) {
            const or_vec8 *v = &regs[r][i];
            wr32(out, cursor, ((u32)(i32)v->dx << 16) | (u32)(uint16_t)v->dy);
            wr32(out, cursor + 4, (v->score & 0x00FFFFFFu) | ((u32)v->luma << 24));
            cursor += 8;
        }
    }
}

void or_pack_vdata_header(const or_analyse_opts *o, int32_t h[16]) { /* :2813-2841 */
    i32 bw, bh, ox, oy, gw, gh;
    or_output_block(o, &bw, &bh, &ox, &oy);
    or_grid(o, bw, bh, ox, oy, &gw, &gh);
    memset(h, 0, 16 * sizeof(i32));
    h[0] = 0xA0; h[1] = o->vectors == 1 ? 1 : (o->vectors == 2 ? 2 : 3); h[2] = bw; h[3] = bh; h[4] = o->pel;
    h[5] = o->has_refine_thsad ? 1 : o->levels; h[7] = o->width; h[8] = o->height; h[9] = ox; h[10] = oy;
    h[11] = gw; h[12] = gh; h[13] = o->selector; h[14] = o->delta;
}

static void portable_planes(const or_super_opts *so, const px *buf, or_planes *p) { /* SuperFrame::planes */
    usize w = (usize)so->width, sh = (usize)or_super_height(so), cw = w / 2;
    usize ylen = w * sh, clen = cw * (sh / 2);
    p->y = buf; p->y_len = ylen; p->y_stride = w;
    p->u = buf + ylen; p->u_len = clen; p->u_stride = cw;
    p->v = buf + ylen + clen; p->v_len = clen; p->v_stride = cw;
    p->luma_w = w; p->luma_h = (usize)so->height; p->pel = so->pel; p->levels = so->levels; p->full = so->full;
}

int or_analyse_portable(const or_analyse_opts *o, const or_super_opts *so, const px *cur_super,
                        const px *ref_super, uint8_t *payload) {
    or_planes a, b;
    portable_planes(so, cur_super, &a);
    portable_planes(so, ref_super, &b);
    i32 bw, bh, ox, oy, gw, gh;
    or_output_block(o, &bw, &bh, &ox, &oy);
    or_grid(o, bw, bh, ox, oy, &gw, &gh);
    usize n = (usize)(gw * gh);
    or_vec8 *bwd = (o->vectors & 1) ? calloc(n, sizeof(or_vec8)) : NULL;
    or_vec8 *fwd = (o->vectors & 2) ? calloc(n, sizeof(or_vec8)) : NULL;
    int rc = or_analyse_pair(&a, &b, o, bwd, fwd);
    if (rc == 0) or_pack_vector_frame(o, bwd, fwd, payload);
    free(bwd);
    free(fwd);
    return rc;
}

int or_analyse_clip(const or_analyse_opts *o, const or_super_opts *so, const px *const *supers, int32_t nframes,
                    int32_t first, int32_t count, uint8_t *payloads, int32_t threads) {
    usize plen = or_payload_len(o);
    i32 delta = imax(o->delta, 1);
    int rc = 0;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads > 0 ? threads : 1) reduction(| : rc)
#endif
    for (i32 k = 0; k < count; k++) {
        i32 n = first + k;
        i32 n2 = imin(n + delta, nframes - 1);
        rc |= or_analyse_portable(o, so, supers[n], supers[n2], payloads + (usize)k * plen);
    }
    (void)threads;
    return rc;
}

/* ------------------------------------------------------------------ svpflow-core consumers */
/* metadata.rs:241-244 extended_grid */
static int32_t ext_grid(int32_t block, int32_t overlap, int32_t grid, int32_t source) {
    i64 span = (i64)(block - overlap) * grid + overlap;
    return grid + (span < source ? 1 : 0);
}
void or_vector_grid(const int32_t vdata[16], int32_t *mw, int32_t *mh) {
    *mw = ext_grid(vdata[2], vdata[9], vdata[11], vdata[7]);
    *mh = ext_grid(vdata[3], vdata[10], vdata[12], vdata[8]);
}
static int rd_i32(const uint8_t *p, size_t len, size_t off, int32_t *v) { /* read_i32_slice, :498-502 */
    if (off > len || len - off < 4) return 0;
    memcpy(v, p + off, 4);
    return 1;
}
/* decode_region (:455-481): 0 when the region does not decode */
/* score / luma: NULL, or the vectors' 24-bit scores and luma bytes (DecodedVector::score, ::luma) */
static int decode_region(const uint8_t *p, size_t len, size_t off, size_t count, int16_t *dx, int16_t *dy,
                         uint32_t *score, uint8_t *luma) {
    int32_t m;
    if (!rd_i32(p, len, off, &m) || (i64)m != (i64)(2 * count + 1)) return 0;
    for (size_t i = 0; i < count; i++) {
        int32_t r0, r1;
        if (!rd_i32(p, len, off + 4 + i * 8, &r0) || !rd_i32(p, len, off + 8 + i * 8, &r1)) return 0;
        uint32_t rot = ((uint32_t)r0 >> 16) | ((uint32_t)r0 << 16); /* rotate_right(16) */
        dx[i] = (int16_t)(rot & 0xFFFF);
        dy[i] = (int16_t)(rot >> 16);
        if (score) score[i] = (uint32_t)r1 & 0x00FFFFFFu;
        if (luma) luma[i] = (uint8_t)((uint32_t)r1 >> 24);
    }
    return 1;
}
static int clamp_frame(int v, int pos, int block, int frame) { /* renderer.rs:1728-1736 */
    if (v + pos < 0) return -pos;
    if (v + block + pos > frame) return imax(frame - block - pos, 0);
    return v;
}
static uint16_t centered16(int v) { return (v > 1023 || v < -1023) ? 1024 : (uint16_t)(v + 1024); } /* :3237-3243 */
/* decode_vectors (metadata.rs:246-273) with SmoothFps' fallbacks (svpflow2 core.rs:962-1001) and
 * vector_planes (renderer.rs:1680-1726) for both sets: out = mvx0 | mvy0 | mvx1 | mvy1. */
int or_vector_planes(const int32_t vdata[16], const uint8_t *p, size_t len, int32_t frame_w, int32_t frame_h,
                     int32_t raw, uint16_t *out) {
    int32_t flags = vdata[1], gw = imax(vdata[11], 0), gh = imax(vdata[12], 0), v;
    if (vdata[0] != 0xA0) return -1;
    if (!rd_i32(p, len, 0, &v) || v != 16 || !rd_i32(p, len, 4, &v) || v != 0xA0 || !rd_i32(p, len, 8, &v) ||
        v != flags)
        return -1;
    size_t count = (size_t)gw * (size_t)gh, first = 0x40, second = first + 4 + count * 8;
    int16_t *pvx = calloc(count + 1, 2), *pvy = calloc(count + 1, 2), *cx = calloc(count + 1, 2),
            *cy = calloc(count + 1, 2);
    int okp = (flags & 1) ? decode_region(p, len, first, count, pvx, pvy, NULL, NULL) : 0;
    int okc = (flags & 2) ? decode_region(p, len, second, count, cx, cy, NULL, NULL) : 0;
    int rc = 0;
    if (((flags & 1) && !okp) || ((flags & 2) && !okc) || (!okp && !okc)) rc = -1;
    else {
        if (!okp) { memcpy(pvx, cx, count * 2); memcpy(pvy, cy, count * 2); }
        if (!okc) { memcpy(cx, pvx, count * 2); memcpy(cy, pvy, count * 2); }
        int32_t mw, mh;
        or_vector_grid(vdata, &mw, &mh);
        mw = imax(mw, 0); mh = imax(mh, 0);
        int32_t bw = imax(vdata[2], 1), bh = imax(vdata[3], 1), stx = bw - vdata[9], sty = bh - vdata[10];
        size_t n = (size_t)mw * (size_t)mh;
        for (int32_t y = 0; y < mh; y++)
            for (int32_t x = 0; x < mw; x++) {
                size_t sx = (size_t)imin(x, imax(gw - 1, 0)), sy = (size_t)imin(y, imax(gh - 1, 0));
                size_t si = sy * (size_t)gw + sx, o = (size_t)y * mw + x;
                for (int w = 0; w < 2; w++) {
                    int dx = 0, dy = 0;
                    if (si < count) { dx = w ? cx[si] : pvx[si]; dy = w ? cy[si] : pvy[si]; }
                    uint16_t ox, oy;
                    if (dx > 1023 || dx < -1023 || dy > 1023 || dy < -1023) ox = oy = 1024;
                    else {
                        if (!raw) { dx = clamp_frame(dx, x * stx, bw, frame_w); dy = clamp_frame(dy, y * sty, bh, frame_h); }
                        ox = centered16(dx); oy = centered16(dy);
                    }
                    out[(size_t)(2 * w) * n + o] = ox;
                    out[(size_t)(2 * w + 1) * n + o] = oy;
                }
            }
    }
    free(pvx); free(pvy); free(cx); free(cy);
    return rc;
}

/* ------------------------------------------------------------------ SmoothFps mask planes */
/* The masks SmoothFps derives from one payload's vectors (svpflow2 core.rs:1154-1195 magnitude,
 * :1467-1499 coverage, :1605-1616 max_mask), for the VectorContext it builds there: block
 * max(bw, 1) x max(bh, 1), origin = the overlap, scale base = max(marker, 1), the payload's grid,
 * planes of the motion grid's size. Restated from renderer.rs: magnitude_mask (:1647-1678),
 * coverage_mask (:1738-1763), splat_coverage (:2945-3062), window_3x3 (:3064-3100),
 * finish_coverage (:3102-3134), add_point (:3136-3147), TruncDiv (:3149-3184), scale_magnitude /
 * clamp_u8 (:3245-3260), coverage_byte (:3262-3273), max_mask (:2908-2915).
 * TruncDiv::div(v) = v / d truncated for every v: for d > 0 and |v| < 2^40 / d the magic product
 * (|v| * ceil(2^40 / d)) >> 40 overshoots |v| / d by |v| * e / (d * 2^40) with e < d, less than 1 / d,
 * so the floor is the exact quotient; elsewhere it divides. */
typedef struct { i32 bw, bh, base, ox, oy, gw, gh; } or_mctx;
static i32 m_div(i32 v, i32 d) { return d == 0 ? 0 : (d == -1 ? (i32)(0u - (u32)v) : v / d); }
static void m_add_point(i32 *acc, usize len, i32 width, i32 x, i32 y, i32 w) {
    if (x < 0 || y < 0) return;
    usize i = sat_add_us(sat_mul_us((usize)y, (usize)width + 2), (usize)x);
    if (i < len) acc[i] = sat_add_i32(acc[i], w);
}
static void m_splat(const or_mctx *c, const int16_t *vdx, const int16_t *vdy, i32 *acc, usize len, i32 w, i32 h,
                    i32 threshold) {
    if (c->gw <= 0 || c->gh <= 0 || w <= 0 || h <= 0) return;
    i32 xs = sat_i64_to_i32((i64)c->bw - c->ox), ys = sat_i64_to_i32((i64)c->bh - c->oy);
    i32 denom = (i32)((u32)c->base << 8);
    if (xs == 0 || ys == 0 || denom == 0) return;
    i32 xb = sat_i64_to_i32((i64)1 - xs), yb = sat_i64_to_i32((i64)1 - ys);
    usize stride = (usize)w + 2;
    for (i32 y = 0; y < c->gh; y++) {
        i32 x_base = 0;
        for (i32 x = 0; x < c->gw; x++) {
            usize k = (usize)y * (usize)c->gw + (usize)x;
            i32 dx = m_div((i32)((u32)threshold * (u32)(i32)vdx[k]), denom);
            i32 dy = m_div((i32)((u32)threshold * (u32)(i32)vdy[k]), denom);
            i32 sx = sat_add_i32(x_base, dx), sy = sat_add_i32(sat_mul_i32(ys, y), dy);
            i32 left = m_div(sx + (xb & (sx >> 31)), xs), top = m_div(sy + (yb & (sy >> 31)), ys);
            i32 right = left + 1, bottom = top + 1;
            i32 next_x = sat_mul_i32(right, xs);
            i32 lw = next_x - sx, tw = sat_mul_i32(ys, bottom) - sy, rw = sx + c->bw - next_x, bw = c->bh - tw;
            int interior = left >= 0 && right < w && top >= 0 && bottom < h;
            usize base = interior ? sat_add_us(sat_mul_us((usize)top, stride), (usize)left) : 0;
            if (interior && sat_add_us(sat_add_us(base, stride), 2) <= len) {
                acc[base] += lw * tw;
                acc[base + 1] += tw * rw;
                acc[base + stride] += lw * bw;
                acc[base + stride + 1] += rw * bw;
            } else {
                if (top >= 0 && top < h && left >= 0 && left < w) m_add_point(acc, len, w, left, top, sat_mul_i32(lw, tw));
                if (left >= -1 && top >= 0 && top < h && right < w) m_add_point(acc, len, w, right, top, sat_mul_i32(tw, rw));
                if (top >= -1 && bottom < h && left >= -1 && right < w)
                    m_add_point(acc, len, w, right, bottom, sat_mul_i32(rw, bw));
                if (left >= 0 && top >= -1 && bottom < h && left < w)
                    m_add_point(acc, len, w, left, bottom, sat_mul_i32(lw, bw));
            }
            x_base = sat_add_i32(x_base, xs);
        }
    }
}
static void m_window3x3(const i32 *pt, i32 *sums, usize stride, usize len) {
    usize rows = len / stride;
    for (usize r = 0; r < rows; r++) {
        const i32 *s = pt + r * stride;
        i32 *o = sums + r * stride;
        o[0] = s[0];
        o[1] = s[1] + s[0];
        for (usize x = 2; x < stride; x++) o[x] = s[x] + s[x - 1] + s[x - 2];
    }
    for (usize y = rows; y-- > 1;) {
        i32 *cur = sums + y * stride;
        const i32 *r1 = sums + (y - 1) * stride, *r2 = y >= 2 ? sums + (y - 2) * stride : NULL;
        for (usize x = 0; x < stride; x++) cur[x] += r1[x] + (r2 ? r2[x] : 0);
    }
}
static uint8_t m_coverage_byte(double v) {
    if (!isfinite(v)) return 0;
    i32 i = f64_as_i32(v);
    return i >= 255 ? 255 : (uint8_t)(i & 0xFF);
}
static uint8_t m_clamp_u8(double v) {
    if (!isfinite(v) || v <= 0.0) return 0;
    if (v >= 255.0) return 255;
    return (uint8_t)v;
}
static void m_coverage(const or_mctx *c, const int16_t *vdx, const int16_t *vdy, uint8_t *out, i32 w, i32 h,
                       i32 strength_percent, i32 threshold) {
    usize stride = (usize)w + 2, len = stride * ((usize)h + 2);
    i32 *pt = calloc(len + 1, sizeof(i32)), *sums = calloc(len + 1, sizeof(i32));
    m_splat(c, vdx, vdy, pt, len, w, h, threshold);
    m_window3x3(pt, sums, stride, len);
    i32 area = imax(sat_mul_i32(c->bw, c->bh), 1);
    double strength = (double)strength_percent / 100.0, area_f = (double)area;
    for (i32 y = 0; y < h; y++)
        for (i32 x = 0; x < w; x++) {
            i32 covered = sums[(usize)(y + 1) * stride + (usize)x + 1] >> 3;
            i32 remaining = area <= covered ? 0 : area - covered;
            out[(usize)y * (usize)w + (usize)x] = m_coverage_byte((double)remaining * strength * 256.0 / area_f);
        }
    free(pt);
    free(sums);
}
static void m_magnitude(const or_mctx *c, const uint32_t *score, uint8_t *out, i32 w, i32 h, double scale,
                        double exponent) {
    i32 area = imax(sat_mul_i32(c->bw, c->bh), 1);
    for (i32 y = 0; y < h; y++)
        for (i32 x = 0; x < w; x++) {
            usize i = (usize)y * (usize)w + (usize)x;
            if (x < c->gw && y < c->gh)
                out[i] = m_clamp_u8(pow(4.0 * (double)score[(usize)y * (usize)c->gw + (usize)x] * scale / (double)area,
                                        exponent) * 255.0);
            else if (x > 0) out[i] = out[i - 1];
            else if (y > 0) out[i] = out[i - (usize)w];
            else out[i] = 0;
        }
}
int or_render_masks(const int32_t vdata[16], const uint8_t *p, size_t len, int32_t phase, int32_t cover,
                    double area_scale, double area_sharp, uint8_t *out) {
    int32_t flags = vdata[1], gw = imax(vdata[11], 0), gh = imax(vdata[12], 0), v;
    if (vdata[0] != 0xA0) return -1;
    if (!rd_i32(p, len, 0, &v) || v != 16 || !rd_i32(p, len, 4, &v) || v != 0xA0 || !rd_i32(p, len, 8, &v) ||
        v != flags)
        return -1;
    size_t count = (size_t)gw * (size_t)gh, first = 0x40, second = first + 4 + count * 8;
    int16_t *vx[2], *vy[2];
    uint32_t *sc[2];
    int ok[2];
    for (int s = 0; s < 2; s++) {
        vx[s] = calloc(count + 1, 2); vy[s] = calloc(count + 1, 2); sc[s] = calloc(count + 1, 4);
    }
    ok[0] = (flags & 1) ? decode_region(p, len, first, count, vx[0], vy[0], sc[0], NULL) : 0;
    ok[1] = (flags & 2) ? decode_region(p, len, second, count, vx[1], vy[1], sc[1], NULL) : 0;
    int rc = 0;
    if (((flags & 1) && !ok[0]) || ((flags & 2) && !ok[1]) || (!ok[0] && !ok[1])) rc = -1;
    else {
        for (int s = 0; s < 2; s++)
            if (!ok[s]) { /* previous falls back to current and vice versa */
                memcpy(vx[s], vx[1 - s], count * 2); memcpy(vy[s], vy[1 - s], count * 2); memcpy(sc[s], sc[1 - s], count * 4);
            }
        int32_t mw, mh;
        or_vector_grid(vdata, &mw, &mh);
        mw = imax(mw, 0); mh = imax(mh, 0);
        or_mctx c = {imax(vdata[2], 1), imax(vdata[3], 1), imax(vdata[4], 1), vdata[9], vdata[10], gw, gh};
        size_t n = (size_t)mw * (size_t)mh;
        /* coverage of mask 0 splats the current set at 256 - phase, mask 1 the previous set at phase */
        m_coverage(&c, vx[1], vy[1], out, mw, mh, cover, 256 - phase);
        m_coverage(&c, vx[0], vy[0], out + n, mw, mh, cover, phase);
        m_magnitude(&c, sc[0], out + 2 * n, mw, mh, area_scale, area_sharp);
        m_magnitude(&c, sc[1], out + 3 * n, mw, mh, area_scale, area_sharp);
        for (size_t i = 0; i < n; i++) out[4 * n + i] = out[2 * n + i] > out[3 * n + i] ? out[2 * n + i] : out[3 * n + i];
    }
    for (int s = 0; s < 2; s++) { free(vx[s]); free(vy[s]); free(sc[s]); }
    return rc;
}

/* ------------------------------------------------------------------ SmoothFps scene class */
/* SmoothFps's scene class of one payload (svpflow2 core.rs:2079-2100): metadata.rs analyze_scene
 * (:349-361) = luma_map (:275-297, with luma_byte :523-526) over the previous / current sets (each
 * falling back to the other) and classify_scene (:299-347) over the current set. */
static uint8_t sc_luma_byte(double value, double gamma) {
    const i32 scaled = f64_as_i32(pow(value, gamma) * 255.0);
    return (uint8_t)((scaled > 20 ? scaled : 20) & 0xFF);
}
int32_t or_scene_class(const int32_t vdata[16], const uint8_t *p, size_t len, double gamma, int32_t blocks_pct,
                       int32_t zero, int32_t m1, int32_t m2, int32_t scene) {
    int32_t flags = vdata[1], gw = imax(vdata[11], 0), gh = imax(vdata[12], 0), v;
    if (vdata[0] != 0xA0) return -1;
    if (!rd_i32(p, len, 0, &v) || v != 16 || !rd_i32(p, len, 4, &v) || v != 0xA0 || !rd_i32(p, len, 8, &v) ||
        v != flags)
        return -1;
    size_t count = (size_t)gw * (size_t)gh, first = 0x40, second = first + 4 + count * 8;
    int16_t *dx = calloc(count + 1, 2), *dy = calloc(count + 1, 2);
    uint32_t *sc[2] = {calloc(count + 1, 4), calloc(count + 1, 4)};
    uint8_t *lu[2] = {calloc(count + 1, 1), calloc(count + 1, 1)}, *map = calloc(count + 1, 1);
    int okp = (flags & 1) ? decode_region(p, len, first, count, dx, dy, sc[0], lu[0]) : 0;
    int okc = (flags & 2) ? decode_region(p, len, second, count, dx, dy, sc[1], lu[1]) : 0;
    int32_t cls;
    if (((flags & 1) && !okp) || ((flags & 2) && !okc)) cls = -1;   /* decode_vectors -> None */
    else if (!okp && !okc) cls = 3;                                  /* no set: scene_class returns 3 */
    else {
        const int ip = okp ? 0 : 1, ic = okc ? 1 : 0;               /* the fallbacks */
        const double denom = vdata[4] == 3 ? 510.0 : 255.0;
        for (size_t i = 0; i < count; i++)
            map[i] = sc_luma_byte(((double)lu[ip][i] + (double)lu[ic][i]) / denom, gamma);
        i32 scene_n = 0, m2_n = 0, m1_n = 0, considered = 0;
        for (i32 y = 0; y < gh; y++)
            for (i32 x = 0; x < gw; x++) {
                const size_t i = (size_t)y * (size_t)gw + (size_t)x;
                const i32 l = imax((i32)map[i], 1);
                const i32 score = sat_mul_i32((i32)sc[ic][i], 255) / l;
                if (score < zero) continue;
                considered++;
                if (score >= scene) scene_n++;
                else if (score >= m2) m2_n++;
                else if (score >= m1) m1_n++;
            }
        const i32 required = (i32)((u32)considered * (u32)blocks_pct) / 100;
        const i32 high = scene_n + m2_n, mid = high + m1_n;
        cls = scene_n >= required ? 3 : (high >= required ? 2 : (mid >= required ? 1 : 0));
    }
    free(dx); free(dy); free(sc[0]); free(sc[1]); free(lu[0]); free(lu[1]); free(map);
    return cls;
}

/* ------------------------------------------------------------------ SmoothFps single-warp render */
/* crates/svpflow-core/src/renderer.rs, 8-bit samples: CpuRenderer::render_mode1_or_2 (:308-328)
 * through render_selected_warp_rows (:876-984) without masks, with its helpers: cpu_map
 * (:3186-3193), set_threshold (:238-250), plane_params (:1539-1606), motion_samples
 * (:1608-1638), render_tiles (:1925-2010), interpolate_row / interpolate_motion_row /
 * interpolate_motion (:2582-2637), interp_pair (:2724-2738), interpolation_weights / coeff
 * (:2740-2770), plane_covers / plane_index / plane_index_checked (:2772-2803), tile_interior
 * (:2809-2835), sample_plane (:2837-2861), output_row (:2894-2906). The scalar loop is the
 * definition followed here. On x86-64 the reference takes its SSE warp_tile (:2090-2349) for
 * interpolated tiles instead: it multiplies the vertical pass in wrapping 16-bit lanes and keeps
 * the low 16 bits of the horizontal result, which equals the 32-bit scalar arithmetic whenever
 * |motion| <= 1024 and the weights are <= 32 (LUT entries are trunc((-1024..1023) * t / 256), so
 * every threshold in 0..256 stays within it). */
#ifndef OR_PX16
static const int32_t r_cpu_map[32] = {0, 1, 2, 2, -1, 3, 3, 3, -1, -1, -1, 4, -1, 4, -1, 4,
                                      -1, -1, -1, -1, -1, -1, -1, -1, 5, -1, -1, -1, 5, -1, -1, 5};
static int32_t r_map(int32_t v) {
    int64_t i = (int64_t)v - 1;
    return (i >= 0 && i < 32) ? r_cpu_map[i] : -1;
}
static int16_t r_div256(int32_t v) {
    int32_t q = v / 256;
    return (int16_t)(q < -32768 ? -32768 : (q > 32767 ? 32767 : q));
}
void or_render_luts(int32_t threshold, int16_t inverse_lut[2048], int16_t threshold_lut[2048]) {
    int32_t inverse = sat_i64_to_i32((int64_t)256 - threshold);
    for (int32_t k = 0; k < 2048; k++) {
        int32_t sample = k - 1024;
        inverse_lut[k] = r_div256(sat_mul_i32(sample, inverse));
        threshold_lut[k] = r_div256(sat_mul_i32(sample, threshold));
    }
}

typedef struct {
    i32 width, height, block_w, block_h, origin_x, origin_y, x_shift, y_shift, x_div, y_div, step, max_x, max_y;
    i32 xw[32][2], yw[32][2];
} rparams;

static void r_weights(i32 total, i32 shift, i32 w[32][2]) {
    memset(w, 0, sizeof(i32) * 64);
    if (total <= 0) return;
    i32 scale = (shift < 0 ? 0 : shift) >= 32 ? 0 : (i32)(1u << (shift < 0 ? 0 : shift));
    for (i32 p = 0; p < total && p < 32; p++) {
        if (shift < 0) { w[p][0] = total - p; w[p][1] = p; }
        else if (scale == 0) { w[p][0] = 1; w[p][1] = 0; }
        else {
            w[p][0] = f64_as_i32(ceil((double)(i32)((u32)(total - p) * (u32)scale) / (double)total - 0.5));
            w[p][1] = f64_as_i32(ceil((double)(i32)((u32)p * (u32)scale) / (double)total - 0.5));
        }
    }
}
static i32 r_satsub1_max0(i32 a, i32 b) { /* a.saturating_mul(b).saturating_sub(1).max(0) */
    i32 m = sat_mul_i32(a, b);
    i32 s = sat_i64_to_i32((int64_t)m - 1);
    return s > 0 ? s : 0;
}
static void r_params(const or_render_config *c, int chroma, int zero_origin, rparams *p) {
    i32 cd = c->chroma_y_div;
    p->origin_x = zero_origin ? 0 : (chroma ? c->origin_x / 2 : c->origin_x);
    p->origin_y = zero_origin ? 0 : (chroma ? c->origin_y / cd : c->origin_y);
    p->step = c->source_step;
    if (chroma) {
        p->width = c->width / 2; p->height = c->height / cd;
        p->block_w = c->block_w / 2; p->block_h = c->block_h / cd;
        p->x_shift = r_map(c->block_w / 2); p->y_shift = r_map(c->block_h / 2);
        p->x_div = 2; p->y_div = cd;
        p->max_x = r_satsub1_max0(c->width / 2, c->source_step);
        p->max_y = r_satsub1_max0(c->height / cd, c->source_step);
        r_weights(c->block_w / 2, p->x_shift, p->xw);
        r_weights(c->block_h / cd, p->y_shift, p->yw);
    } else {
        p->width = c->width; p->height = c->height;
        p->block_w = c->block_w; p->block_h = c->block_h;
        p->x_shift = r_map(c->block_w); p->y_shift = r_map(c->block_h);
        p->x_div = 1; p->y_div = 1;
        p->max_x = r_satsub1_max0(c->width, c->source_step);
        p->max_y = r_satsub1_max0(c->height, c->source_step);
        r_weights(c->block_w, p->x_shift, p->xw);
        r_weights(c->block_h, p->y_shift, p->yw);
    }
}
static usize r_index(const or_rplane *pl, usize x, usize y) {
    if (pl->shift == 0) return y * pl->stride + x;
    usize mask = ((usize)1 << pl->shift) - 1;
    usize sub = ((y & mask) << pl->shift) | (x & mask);
    return sub * pl->span + (y >> pl->shift) * pl->stride + (x >> pl->shift);
}
static int r_covers(const or_rplane *pl, const rparams *p) {
    if (pl->shift != 0 && (pl->shift >= 32 || (i32)(1u << pl->shift) != p->step)) return 0;
    usize x = (usize)p->max_x, y = (usize)p->max_y;
    unsigned __int128 idx;
    if (pl->shift == 0) idx = (unsigned __int128)y * pl->stride + x;
    else {
        usize mask = ((usize)1 << pl->shift) - 1;
        usize sub = ((y & mask) << pl->shift) | (x & mask);
        idx = (unsigned __int128)sub * pl->span + (unsigned __int128)(y >> pl->shift) * pl->stride + (x >> pl->shift);
    }
    return idx < (unsigned __int128)pl->len;
}
static i32 r_interp(i32 a, i32 b, i32 total, i32 shift, const i32 w[2]) {
    i32 s = (i32)((u32)w[0] * (u32)a + (u32)w[1] * (u32)b);
    if (shift < 0) return total ? s / total : 0;
    return s >> shift;
}
static i32 r_motion(const int16_t *lut, const uint16_t *plane, usize len, usize i) {
    usize k = i < len ? plane[i] : 1024;
    return lut[k < 2047 ? k : 2047];
}

/* alpha_at_absolute (:2687-2722) and mask_at (:3209-3219) */
static i32 r_mask_at(const uint8_t *m, usize len, usize stride, i32 x, i32 y) {
    if (x < 0 || y < 0) return 0;
    usize i = sat_add_us(sat_mul_us((usize)y, stride), (usize)x);
    return i < len ? m[i] : 0;
}
static i32 r_byte(i32 v) { return v < 0 ? 0 : (v > 255 ? 255 : v); }
static i32 r_alpha_abs(const uint8_t *m, usize len, const rparams *q, usize stride, i32 x, i32 y) {
    if (q->block_w <= 0 || q->block_h <= 0) return 0;
    i32 ix0 = 0, ix1 = 0, iy0 = 0, iy1 = 0;
    if (q->origin_x <= x) { ix0 = (x - q->origin_x) / q->block_w; ix1 = ix0 + 1; }
    if (q->origin_y <= y) { iy0 = (y - q->origin_y) / q->block_h; iy1 = iy0 + 1; }
    i32 fx = q->origin_x < x ? (x - q->origin_x) % q->block_w : 0;
    i32 fy = q->origin_y < y ? (y - q->origin_y) % q->block_h : 0;
    i32 tl = r_mask_at(m, len, stride, ix0, iy0), tr = r_mask_at(m, len, stride, ix1, iy0);
    i32 bl = r_mask_at(m, len, stride, ix0, iy1), br = r_mask_at(m, len, stride, ix1, iy1);
    i32 top = ((q->block_w - fx) * tl + fx * tr) / q->block_w;
    i32 bottom = ((q->block_w - fx) * bl + fx * br) / q->block_w;
    return r_byte(((q->block_h - fy) * top + fy * bottom) / q->block_h);
}

void or_render_warp_plane(const or_render_config *c, int32_t chroma, int32_t interp, const int16_t *lut,
                          const or_rplane *src, const uint16_t *mx, const uint16_t *my, size_t mlen,
                          const uint8_t *mask, uint8_t *dst, size_t dst_stride, size_t dst_len) {
    rparams P, MP;
    r_params(c, chroma, !interp, &P);
    r_params(c, chroma, 0, &MP); /* mask_params: the plane's own origin, used without interpolation */
    const rparams *p = &P;
    i32 gw = (i32)c->grid_w, gh = (i32)c->grid_h;
    if (p->width <= 0 || p->height <= 0 || p->block_w <= 0 || p->block_h <= 0 || gw <= 0 || gh <= 0) return;
    i32 rows_end = chroma ? c->height / c->chroma_y_div : c->height;
    for (i32 gy = -1; gy < gh; gy++) {
        i32 base_y = gy < 0 ? 0 : p->origin_y + p->block_h * gy;
        i32 height = gy < 0 ? p->origin_y : p->block_h;
        if (base_y + p->block_h >= p->height || gy == gh - 1) height = p->height - base_y;
        i32 end_y = base_y + height < rows_end ? base_y + height : rows_end;
        i32 clipped_y = base_y > 0 ? base_y : 0;
        height = end_y - clipped_y;
        if (height <= 0) continue;
        for (i32 gx = -1; gx < gw; gx++) {
            i32 base_x = gx < 0 ? 0 : p->origin_x + p->block_w * gx;
            i32 width = gx < 0 ? p->origin_x : p->block_w;
            if (base_x + p->block_w >= p->width || gx == gw - 1) width = p->width - base_x;
            if (width <= 0) continue;
            usize x0 = (usize)(gx > 0 ? gx : 0), y0 = (usize)(gy > 0 ? gy : 0);
            usize nx = (gx >= 0 && gx != gw - 1) ? 1 : 0, ny = (gy >= 0 && gy != gh - 1) ? (usize)gw : 0;
            usize i00 = y0 * (usize)gw + x0, i01 = i00 + nx, i10 = i00 + ny, i11 = i00 + ny + nx;
            i32 tx = base_x, ty = clipped_y, local_y0 = clipped_y - base_y;
            /* motion_samples */
            i32 sx[4], sy[4];
            sx[0] = r_motion(lut, mx, mlen, i00) / p->x_div;
            sy[0] = r_motion(lut, my, mlen, i00) / p->y_div;
            if (!interp) { for (int q = 1; q < 4; q++) { sx[q] = sx[0]; sy[q] = sy[0]; } }
            else {
                usize ii[4] = {i00, i01, i10, i11};
                for (int q = 1; q < 4; q++) {
                    sx[q] = r_motion(lut, mx, mlen, ii[q]) / p->x_div;
                    sy[q] = r_motion(lut, my, mlen, ii[q]) / p->y_div;
                }
            }
            int covers = r_covers(src, p);
            int direct = 0;
            if (covers && p->step > 0) { /* tile_interior */
                i32 mnx = INT32_MAX, mxx = INT32_MIN, mny = INT32_MAX, mxy = INT32_MIN;
                for (int q = 0; q < 4; q++) {
                    mnx = sx[q] < mnx ? sx[q] : mnx; mxx = sx[q] > mxx ? sx[q] : mxx;
                    mny = sy[q] < mny ? sy[q] : mny; mxy = sy[q] > mxy ? sy[q] : mxy;
                }
                int64_t st = p->step;
                direct = (int64_t)tx * st + mnx >= 0 && (int64_t)ty * st + mny >= 0 &&
                         (int64_t)(tx + width - 1) * st + mxx <= p->max_x && (int64_t)(ty + height - 1) * st + mxy <= p->max_y;
            }
            for (i32 y = 0; y < height; y++) {
                i32 local_y = local_y0 + y;
                i32 source_y = (ty + y) * p->step;
                usize row = (usize)(ty + y); /* row_start = 0 */
                usize start = row * dst_stride + (usize)tx;
                if (start + (usize)width > dst_len) continue; /* output_row */
                i32 rx[2], ry[2];
                if (!interp) { rx[0] = rx[1] = sx[0]; ry[0] = ry[1] = sy[0]; }
                else {
                    const i32 *wy = p->yw[local_y < 0 ? 0 : (local_y > 31 ? 31 : local_y)];
                    rx[0] = r_interp(sx[0], sx[2], p->block_h, p->y_shift, wy);
                    rx[1] = r_interp(sx[1], sx[3], p->block_h, p->y_shift, wy);
                    ry[0] = r_interp(sy[0], sy[2], p->block_h, p->y_shift, wy);
                    ry[1] = r_interp(sy[1], sy[3], p->block_h, p->y_shift, wy);
                }
                i32 mrow[2] = {0, 0}; /* alpha_row (:2639-2651) */
                if (mask) {
                    i32 ma = r_mask_at(mask, mlen, mlen, (i32)i00, 0), mb = r_mask_at(mask, mlen, mlen, (i32)i01, 0);
                    i32 mc = r_mask_at(mask, mlen, mlen, (i32)i10, 0), md = r_mask_at(mask, mlen, mlen, (i32)i11, 0);
                    if (!interp) { mrow[0] = mrow[1] = ma; }
                    else {
                        const i32 *wy = p->yw[local_y < 0 ? 0 : (local_y > 31 ? 31 : local_y)];
                        mrow[0] = r_interp(ma, mc, p->block_h, p->y_shift, wy);
                        mrow[1] = r_interp(mb, md, p->block_h, p->y_shift, wy);
                    }
                }
                for (i32 x = 0; x < width; x++) {
                    i32 px = tx + x, source_x = px * p->step;
                    const i32 *wx = p->xw[x > 31 ? 31 : x];
                    i32 dx = rx[0], dy = ry[0];
                    if (interp) {
                        dx = r_interp(rx[0], rx[1], p->block_w, p->x_shift, wx);
                        dy = r_interp(ry[0], ry[1], p->block_w, p->x_shift, wx);
                    }
                    i32 xs = source_x + dx, ys = source_y + dy;
                    uint8_t v, base = 0;
                    if (mask) { /* sample_plane at no displacement */
                        i32 bxs = source_x, bys = source_y;
                        if (!direct) {
                            bxs = bxs < 0 ? 0 : (bxs > p->max_x ? p->max_x : bxs);
                            bys = bys < 0 ? 0 : (bys > p->max_y ? p->max_y : bys);
                        }
                        usize bi = r_index(src, (usize)(int64_t)bxs, (usize)(int64_t)bys);
                        base = bi < src->len ? src->data[bi] : 0;
                    }
                    if (direct) {
                        usize idx = r_index(src, (usize)(int64_t)xs, (usize)(int64_t)ys);
                        v = idx < src->len ? src->data[idx] : 0; /* in range by tile_interior + plane_covers */
                    } else {
                        xs = xs < 0 ? 0 : (xs > p->max_x ? p->max_x : xs);
                        ys = ys < 0 ? 0 : (ys > p->max_y ? p->max_y : ys);
                        usize idx = r_index(src, (usize)xs, (usize)ys);
                        v = idx < src->len ? src->data[idx] : 0;
                    }
                    if (mask) { /* mode1_pixel (:1818-1820) = blend_255(warped, base, alpha) (:3221-3223) */
                        i32 alpha = interp ? r_byte(r_interp(mrow[0], mrow[1], p->block_w, p->x_shift, wx))
                                           : r_alpha_abs(mask, mlen, &MP, (usize)c->grid_w, px, ty + y);
                        v = (uint8_t)r_byte(((i32)v * (255 - alpha) + (i32)base * alpha + 255) >> 8);
                    }
                    dst[start + (usize)x] = v;
                }
            }
        }
    }
}

/* render_dual_warp_rows (:1031-1172) as render_mode11_or_13 (:330-438, and its zero-origin variant)
 * and render_mode21_or_22 (:571-641) drive it: motion set 0 scaled by the threshold LUT reads source 0,
 * set 1 scaled by the inverse LUT reads source 1. mode 11 / 13: mode11_or_13_pixel (:2918-2943) with
 * max_mask(a, b) (:2908-2915) when the masks are given; mode 21 / 22: mode21_or_22_pixel (:615-641)
 * with alpha0 from mask a, alpha1 from mask b and the final mask blending towards the undisplaced
 * samples at threshold_limit. */
int32_t or_render_threshold_limit(int32_t threshold, double scale) {
    int32_t inverse = sat_i64_to_i32((int64_t)256 - threshold);
    return threshold > 126 ? f64_as_i32(256.0 - (double)inverse * scale) : f64_as_i32((double)threshold * scale);
}
static i32 r_blend256(i32 a, i32 b, i32 w) { return r_byte((a * (256 - w) + b * w) >> 8); }
static i32 r_alpha(const uint8_t *m, usize mlen, const usize ii[4], const rparams *p, const rparams *mp, usize gw,
                   int interp, int zero_origin, const i32 *wy, const i32 *wx, i32 px, i32 py) {
    if (zero_origin) return r_alpha_abs(m, mlen, mp, gw, px, py);
    i32 v[4];
    for (int q = 0; q < 4; q++) v[q] = ii[q] < mlen ? m[ii[q]] : 0;
    if (!interp) return r_byte(v[0]);
    i32 r0 = r_interp(v[0], v[2], p->block_h, p->y_shift, wy), r1 = r_interp(v[1], v[3], p->block_h, p->y_shift, wy);
    return r_byte(r_interp(r0, r1, p->block_w, p->x_shift, wx));
}
void or_render_dual_plane(const or_render_config *c, int32_t chroma, int32_t interp, int32_t zero_origin,
                          int32_t mode, int32_t threshold, int32_t threshold_limit, const or_rplane *src0,
                          const or_rplane *src1, const uint16_t *mx0, const uint16_t *my0, const uint16_t *mx1,
                          const uint16_t *my1, size_t mlen, const uint8_t *mask_a, const uint8_t *mask_b,
                          const uint8_t *mask_f, uint8_t *dst, size_t dst_stride, size_t dst_len) {
    int32_t mode13 = mode == 13;
    uint8_t *mask = NULL; /* modes 11 / 13: max_mask */
    if ((mode == 11 || mode == 13) && mask_a && mask_b) {
        mask = malloc(mlen ? mlen : 1);
        for (usize i = 0; i < mlen; i++) mask[i] = mask_a[i] > mask_b[i] ? mask_a[i] : mask_b[i];
    }
    int16_t inv[2048], thr[2048];
    or_render_luts(threshold, inv, thr);
    rparams P, MP;
    r_params(c, chroma, zero_origin, &P);
    r_params(c, chroma, 0, &MP);
    const rparams *p = &P;
    i32 gw = (i32)c->grid_w, gh = (i32)c->grid_h;
    if (p->width <= 0 || p->height <= 0 || p->block_w <= 0 || p->block_h <= 0 || gw <= 0 || gh <= 0) return;
    i32 rows_end = chroma ? c->height / c->chroma_y_div : c->height;
    int covers = r_covers(src0, p) && r_covers(src1, p);
    for (i32 gy = -1; gy < gh; gy++) {
        i32 base_y = gy < 0 ? 0 : p->origin_y + p->block_h * gy;
        i32 height = gy < 0 ? p->origin_y : p->block_h;
        if (base_y + p->block_h >= p->height || gy == gh - 1) height = p->height - base_y;
        i32 end_y = base_y + height < rows_end ? base_y + height : rows_end;
        i32 clipped_y = base_y > 0 ? base_y : 0;
        height = end_y - clipped_y;
        if (height <= 0) continue;
        for (i32 gx = -1; gx < gw; gx++) {
            i32 base_x = gx < 0 ? 0 : p->origin_x + p->block_w * gx;
            i32 width = gx < 0 ? p->origin_x : p->block_w;
            if (base_x + p->block_w >= p->width || gx == gw - 1) width = p->width - base_x;
            if (width <= 0) continue;
            usize x0 = (usize)(gx > 0 ? gx : 0), y0 = (usize)(gy > 0 ? gy : 0);
            usize nx = (gx >= 0 && gx != gw - 1) ? 1 : 0, ny = (gy >= 0 && gy != gh - 1) ? (usize)gw : 0;
            usize ii[4] = {y0 * (usize)gw + x0, 0, 0, 0};
            ii[1] = ii[0] + nx; ii[2] = ii[0] + ny; ii[3] = ii[0] + ny + nx;
            i32 tx = base_x, ty = clipped_y;
            i32 sx[2][4], sy[2][4];
            for (int set = 0; set < 2; set++) {
                const int16_t *lut = set ? inv : thr;
                const uint16_t *mx = set ? mx1 : mx0, *my = set ? my1 : my0;
                for (int q = 0; q < 4; q++) {
                    usize i = interp ? ii[q] : ii[0];
                    sx[set][q] = r_motion(lut, mx, mlen, i) / p->x_div;
                    sy[set][q] = r_motion(lut, my, mlen, i) / p->y_div;
                }
            }
            int direct = 0;
            if (covers && p->step > 0) {
                i32 mnx = INT32_MAX, mxx = INT32_MIN, mny = INT32_MAX, mxy = INT32_MIN;
                for (int set = 0; set < 2; set++)
                    for (int q = 0; q < 4; q++) {
                        mnx = sx[set][q] < mnx ? sx[set][q] : mnx; mxx = sx[set][q] > mxx ? sx[set][q] : mxx;
                        mny = sy[set][q] < mny ? sy[set][q] : mny; mxy = sy[set][q] > mxy ? sy[set][q] : mxy;
                    }
                int64_t st = p->step;
                direct = (int64_t)tx * st + mnx >= 0 && (int64_t)ty * st + mny >= 0 &&
                         (int64_t)(tx + width - 1) * st + mxx <= p->max_x && (int64_t)(ty + height - 1) * st + mxy <= p->max_y;
            }
            for (i32 y = 0; y < height; y++) {
                i32 local_y = clipped_y - base_y + y;
                i32 source_y = (ty + y) * p->step;
                usize start = (usize)(ty + y) * dst_stride + (usize)tx;
                if (start + (usize)width > dst_len) continue;
                const i32 *wy = p->yw[local_y < 0 ? 0 : (local_y > 31 ? 31 : local_y)];
                i32 row[2][2][2]; /* set, x/y, left/right */
                for (int set = 0; set < 2; set++) {
                    if (!interp) { row[set][0][0] = row[set][0][1] = sx[set][0]; row[set][1][0] = row[set][1][1] = sy[set][0]; }
                    else {
                        row[set][0][0] = r_interp(sx[set][0], sx[set][2], p->block_h, p->y_shift, wy);
                        row[set][0][1] = r_interp(sx[set][1], sx[set][3], p->block_h, p->y_shift, wy);
                        row[set][1][0] = r_interp(sy[set][0], sy[set][2], p->block_h, p->y_shift, wy);
                        row[set][1][1] = r_interp(sy[set][1], sy[set][3], p->block_h, p->y_shift, wy);
                    }
                }
                i32 mrow[2] = {0, 0};
                if (mask) {
                    i32 m[4];
                    for (int q = 0; q < 4; q++) m[q] = ii[q] < mlen ? mask[ii[q]] : 0;
                    if (!interp) { mrow[0] = mrow[1] = m[0]; }
                    else {
                        mrow[0] = r_interp(m[0], m[2], p->block_h, p->y_shift, wy);
                        mrow[1] = r_interp(m[1], m[3], p->block_h, p->y_shift, wy);
                    }
                }
                for (i32 x = 0; x < width; x++) {
                    i32 px = tx + x, source_x = px * p->step;
                    const i32 *wx = p->xw[x > 31 ? 31 : x];
                    i32 v[2], cur[2];
                    for (int set = 0; set < 2; set++) {
                        const or_rplane *src = set ? src1 : src0;
                        i32 dx = row[set][0][0], dy = row[set][1][0];
                        if (interp) {
                            dx = r_interp(row[set][0][0], row[set][0][1], p->block_w, p->x_shift, wx);
                            dy = r_interp(row[set][1][0], row[set][1][1], p->block_w, p->x_shift, wx);
                        }
                        i32 xs = source_x + dx, ys = source_y + dy, bxs = source_x, bys = source_y;
                        if (!direct) {
                            xs = xs < 0 ? 0 : (xs > p->max_x ? p->max_x : xs);
                            ys = ys < 0 ? 0 : (ys > p->max_y ? p->max_y : ys);
                            bxs = bxs > p->max_x ? p->max_x : bxs;
                            bys = bys > p->max_y ? p->max_y : bys;
                        }
                        usize idx = r_index(src, (usize)(int64_t)xs, (usize)(int64_t)ys);
                        usize bi = r_index(src, (usize)(int64_t)bxs, (usize)(int64_t)bys);
                        v[set] = idx < src->len ? src->data[idx] : 0;
                        cur[set] = bi < src->len ? src->data[bi] : 0;
                    }
                    i32 motion;
                    if (mode == 21 || mode == 22) {
                        i32 a0 = r_alpha(mask_a, mlen, ii, p, &MP, (usize)c->grid_w, interp, zero_origin, wy, wx, px, ty + y);
                        i32 a1 = r_alpha(mask_b, mlen, ii, p, &MP, (usize)c->grid_w, interp, zero_origin, wy, wx, px, ty + y);
                        i32 a = r_byte((v[0] * (255 - a0) + v[1] * a0 + 255) >> 8);
                        i32 b = r_byte((v[1] * (255 - a1) + v[0] * a1 + 255) >> 8);
                        if (mode == 21) motion = r_blend256(a, b, threshold);
                        else {
                            i32 m = r_blend256(cur[0], cur[1], threshold), lo = a < b ? a : b, hi = a < b ? b : a;
                            motion = m < lo ? lo : (m > hi ? hi : m);
                        }
                        if (mask_f) {
                            i32 fa = r_alpha(mask_f, mlen, ii, p, &MP, (usize)c->grid_w, interp, zero_origin, wy, wx, px, ty + y);
                            motion = r_byte((motion * (255 - fa) + r_blend256(cur[0], cur[1], threshold_limit) * fa + 255) >> 8);
                        }
                    } else if (mode13) {
                        i32 b = r_blend256(cur[0], cur[1], threshold);
                        i32 lo = v[0] < v[1] ? v[0] : v[1], hi = v[0] < v[1] ? v[1] : v[0];
                        motion = b < lo ? lo : (b > hi ? hi : b);
                    } else {
                        motion = r_blend256(v[0], v[1], threshold);
                    }
                    if (mask && mode != 21 && mode != 22) {
                        i32 alpha = zero_origin ? r_alpha_abs(mask, mlen, &MP, (usize)c->grid_w, px, ty + y)
                                                : r_byte(interp ? r_interp(mrow[0], mrow[1], p->block_w, p->x_shift, wx)
                                                                : mrow[0]);
                        i32 base = r_blend256(cur[0], cur[1], threshold);
                        motion = r_byte((motion * (255 - alpha) + base * alpha + 255) >> 8);
                    }
                    dst[start + (usize)x] = (uint8_t)motion;
                }
            }
        }
    }
    free(mask);
}

/* render_mode23_plane_rows_inner (:1294-1537) with mode23_pixel (:1850-1868): four motion sets (base0
 * and next0 with the threshold LUT reading source 0, base1 and prev1 with the inverse LUT reading
 * source 1), alphas t0 / t1 from masks a / b, the optional final mask towards blend_256(base_a,
 * base_b, threshold); zero origin when not interpolated. */
void or_render_mode23_plane(const or_render_config *c, int32_t chroma, int32_t interp, int32_t threshold,
                            const or_rplane *src0, const or_rplane *src1, const uint16_t *const mxs[4],
                            const uint16_t *const mys[4], size_t mlen, const uint8_t *mask_a, const uint8_t *mask_b,
                            const uint8_t *mask_f, uint8_t *dst, size_t dst_stride, size_t dst_len) {
    int16_t inv[2048], thr[2048];
    or_render_luts(threshold, inv, thr);
    int zero_origin = !interp;
    rparams P, MP;
    r_params(c, chroma, zero_origin, &P);
    r_params(c, chroma, 0, &MP);
    const rparams *p = &P;
    i32 gw = (i32)c->grid_w, gh = (i32)c->grid_h;
    if (p->width <= 0 || p->height <= 0 || p->block_w <= 0 || p->block_h <= 0 || gw <= 0 || gh <= 0) return;
    i32 rows_end = chroma ? c->height / c->chroma_y_div : c->height;
    int covers = r_covers(src0, p) && r_covers(src1, p);
    for (i32 gy = -1; gy < gh; gy++) {
        i32 base_y = gy < 0 ? 0 : p->origin_y + p->block_h * gy;
        i32 height = gy < 0 ? p->origin_y : p->block_h;
        if (base_y + p->block_h >= p->height || gy == gh - 1) height = p->height - base_y;
        i32 end_y = base_y + height < rows_end ? base_y + height : rows_end;
        i32 clipped_y = base_y > 0 ? base_y : 0;
        height = end_y - clipped_y;
        if (height <= 0) continue;
        for (i32 gx = -1; gx < gw; gx++) {
            i32 base_x = gx < 0 ? 0 : p->origin_x + p->block_w * gx;
            i32 width = gx < 0 ? p->origin_x : p->block_w;
            if (base_x + p->block_w >= p->width || gx == gw - 1) width = p->width - base_x;
            if (width <= 0) continue;
            usize x0 = (usize)(gx > 0 ? gx : 0), y0 = (usize)(gy > 0 ? gy : 0);
            usize nx = (gx >= 0 && gx != gw - 1) ? 1 : 0, ny = (gy >= 0 && gy != gh - 1) ? (usize)gw : 0;
            usize ii[4] = {y0 * (usize)gw + x0, 0, 0, 0};
            ii[1] = ii[0] + nx; ii[2] = ii[0] + ny; ii[3] = ii[0] + ny + nx;
            i32 tx = base_x, ty = clipped_y;
            i32 sx[4][4], sy[4][4];
            for (int set = 0; set < 4; set++) {
                const int16_t *lut = (set & 1) ? inv : thr;
                for (int q = 0; q < 4; q++) {
                    usize i = interp ? ii[q] : ii[0];
                    sx[set][q] = r_motion(lut, mxs[set], mlen, i) / p->x_div;
                    sy[set][q] = r_motion(lut, mys[set], mlen, i) / p->y_div;
                }
            }
            int direct = 0;
            if (covers && p->step > 0) {
                i32 mnx = INT32_MAX, mxx = INT32_MIN, mny = INT32_MAX, mxy = INT32_MIN;
                for (int set = 0; set < 4; set++)
                    for (int q = 0; q < 4; q++) {
                        mnx = sx[set][q] < mnx ? sx[set][q] : mnx; mxx = sx[set][q] > mxx ? sx[set][q] : mxx;
                        mny = sy[set][q] < mny ? sy[set][q] : mny; mxy = sy[set][q] > mxy ? sy[set][q] : mxy;
                    }
                int64_t st = p->step;
                direct = (int64_t)tx * st + mnx >= 0 && (int64_t)ty * st + mny >= 0 &&
                         (int64_t)(tx + width - 1) * st + mxx <= p->max_x && (int64_t)(ty + height - 1) * st + mxy <= p->max_y;
            }
            for (i32 y = 0; y < height; y++) {
                i32 local_y = clipped_y - base_y + y;
                i32 source_y = (ty + y) * p->step;
                usize start = (usize)(ty + y) * dst_stride + (usize)tx;
                if (start + (usize)width > dst_len) continue;
                const i32 *wy = p->yw[local_y < 0 ? 0 : (local_y > 31 ? 31 : local_y)];
                i32 row[4][2][2];
                for (int set = 0; set < 4; set++) {
                    if (!interp) { row[set][0][0] = row[set][0][1] = sx[set][0]; row[set][1][0] = row[set][1][1] = sy[set][0]; }
                    else {
                        row[set][0][0] = r_interp(sx[set][0], sx[set][2], p->block_h, p->y_shift, wy);
                        row[set][0][1] = r_interp(sx[set][1], sx[set][3], p->block_h, p->y_shift, wy);
                        row[set][1][0] = r_interp(sy[set][0], sy[set][2], p->block_h, p->y_shift, wy);
                        row[set][1][1] = r_interp(sy[set][1], sy[set][3], p->block_h, p->y_shift, wy);
                    }
                }
                for (i32 x = 0; x < width; x++) {
                    i32 px = tx + x, source_x = px * p->step;
                    const i32 *wx = p->xw[x > 31 ? 31 : x];
                    i32 v[4];
                    for (int set = 0; set < 4; set++) {
                        const or_rplane *src = (set & 1) ? src1 : src0;
                        i32 dx = row[set][0][0], dy = row[set][1][0];
                        if (interp) {
                            dx = r_interp(row[set][0][0], row[set][0][1], p->block_w, p->x_shift, wx);
                            dy = r_interp(row[set][1][0], row[set][1][1], p->block_w, p->x_shift, wx);
                        }
                        i32 xs = source_x + dx, ys = source_y + dy;
                        if (!direct) {
                            xs = xs < 0 ? 0 : (xs > p->max_x ? p->max_x : xs);
                            ys = ys < 0 ? 0 : (ys > p->max_y ? p->max_y : ys);
                        }
                        usize idx = r_index(src, (usize)(int64_t)xs, (usize)(int64_t)ys);
                        v[set] = idx < src->len ? src->data[idx] : 0;
                    }
                    i32 a = v[0], b = v[1], cc = v[2], d = v[3];
                    i32 t0 = r_alpha(mask_a, mlen, ii, p, &MP, (usize)c->grid_w, interp, zero_origin, wy, wx, px, ty + y);
                    i32 t1 = r_alpha(mask_b, mlen, ii, p, &MP, (usize)c->grid_w, interp, zero_origin, wy, wx, px, ty + y);
                    i32 lo = a < b ? a : b, hi = a < b ? b : a;
                    i32 dcl = d < lo ? lo : (d > hi ? hi : d), ccl = cc < lo ? lo : (cc > hi ? hi : cc);
                    i32 i0 = r_byte((a * (255 - t0) + dcl * t0 + 255) >> 8);
                    i32 i1 = r_byte((b * (255 - t1) + ccl * t1 + 255) >> 8);
                    i32 motion = r_blend256(i0, i1, threshold);
                    if (mask_f) {
                        i32 bxs = source_x > p->max_x ? p->max_x : source_x, bys = source_y > p->max_y ? p->max_y : source_y;
                        usize b0 = r_index(src0, (usize)bxs, (usize)bys), b1 = r_index(src1, (usize)bxs, (usize)bys);
                        i32 ba = b0 < src0->len ? src0->data[b0] : 0, bb = b1 < src1->len ? src1->data[b1] : 0;
                        i32 fa = r_alpha(mask_f, mlen, ii, p, &MP, (usize)c->grid_w, interp, zero_origin, wy, wx, px, ty + y);
                        motion = r_byte((motion * (255 - fa) + r_blend256(ba, bb, threshold) * fa + 255) >> 8);
                    }
                    dst[start + (usize)x] = (uint8_t)motion;
                }
            }
        }
    }
}
#endif
