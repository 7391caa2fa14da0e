// super.cu -- Super pyramid builder on sm_100a (crates/svpflow1/src/super_build.rs).
//
// One launch writes the level-0 region of every plane of every frame (the copied
// plane plus the pel sub-planes), then one launch per pyramid level reduces level l
// into level l+1. Every byte of the output frame is written (zeros where the
// reference leaves its zero-filled frame untouched), so the caller's buffer needs no
// clearing. The reference fills its sub-planes in place, in a fixed loop order, and
// some reads land in bytes an earlier loop wrote; those reads are restated here as
// closed forms of the source plane (see h_val / flat below), which keeps every output
// byte independent and the kernels free of intra-launch dependencies.
//
// HBM-bound streaming work: a frame is read once per level and written once.
//
// The kernels are templates on the sample type: uint8_t is the reference's format; uint16_t
// carries this project's 10-bit extension (samples 0..1023, the same arithmetic with the
// clamps at 1023 instead of 255).
#include <cuda_runtime.h>

#include <algorithm>
#include <stdint.h>

#include "svpf_device.h"

namespace svpf {

namespace {

// Dynamic shared memory the band kernel may take (a band of one row: 7 rows of the level-0 width).
constexpr int64_t kBandSmemMax = 200 << 10;

__device__ __forceinline__ unsigned avg8(unsigned a, unsigned b) { return (a + b + 1u) >> 1; }

struct PlaneGeo {
    int w, h;            // level-0 plane size (chroma: luma/2)
    int64_t stride;      // output row pitch
    int64_t rows;        // output rows that exist in the buffer
    int64_t out_off;     // plane offset inside the output frame
    int64_t src_stride;  // source row pitch
    int64_t src_off;     // plane offset inside the source frame
};

__device__ __forceinline__ PlaneGeo plane_geo(const SuperDev &D, int plane) {
    PlaneGeo g;
    bool c = plane > 0;
    g.w = c ? D.width / 2 : D.width;
    g.h = c ? D.height / 2 : D.height;
    g.stride = c ? D.c_stride : D.y_stride;
    g.rows = c ? D.c_rows : D.y_rows;
    g.out_off = plane == 0 ? 0 : (plane == 1 ? D.y_len : D.y_len + D.c_len);
    g.src_stride = c ? D.src_c_stride : D.src_y_stride;
    g.src_off = plane == 0 ? 0 : (plane == 1 ? D.src_y_len : D.src_y_len + D.src_c_len);
    return g;
}

// Level-0 plane with its row padding: the copy is edge-extended to the pitch
// (super_build.rs:45-67).
template <typename T>
struct L0View {
    const T *s;
    int64_t sst;
    int w, h;
    int64_t stride;
    __device__ __forceinline__ unsigned L(int y, int64_t x) const {
        return s[(int64_t)y * sst + (x < w ? x : (int64_t)w - 1)];
    }
    // byte at flat offset o from the start of the level-0 region, for offsets inside
    // the copied plane (o < h*stride)
    __device__ __forceinline__ unsigned F1(int64_t o) const { return L((int)(o / stride), o % stride); }
    // fill_bilinear_pel2's h-plane value (super_build.rs:185-191). Its right-hand
    // neighbour is the next byte in memory; for the last byte of the plane that is the
    // h-plane's own first byte, already written by then.
    __device__ __forceinline__ unsigned h_val(int y, int x) const {
        int64_t n = (int64_t)y * stride + x + 1;
        unsigned b;
        if (n / stride < h) b = F1(n);
        else b = avg8(L(0, 0), F1(1));
        return avg8(L(y, x), b);
    }
    // any byte of the copied plane or of the h plane that follows it
    __device__ __forceinline__ unsigned flat(int64_t o) const {
        int64_t r = o / stride, c = o % stride;
        if (r < h) return L((int)r, c);
        return c < w ? h_val((int)(r - h), (int)c) : 0u;
    }
};

// half(), super_build.rs:162-177 (cubic8 at :138-160 computes the same value)
template <typename Get>
__device__ __forceinline__ unsigned half_tap(Get g, int p, int n, int pmax) {
    if (p < 2 || p + 4 >= n) return p + 1 == n ? g(p) : avg8(g(p), g(p + 1));
    int v = (int)g(p - 2) + (int)g(p + 3) + 5 * (4 * (int)g(p) - (int)g(p - 1) + 4 * (int)g(p + 1) - (int)g(p + 2)) + 16;
    v >>= 5;
    return (unsigned)(v < 0 ? 0 : (v > pmax ? pmax : v));
}

template <typename T>
__global__ void __launch_bounds__(256) super_level0_kernel(SuperDev D, const T *__restrict__ src,
                                                           T *__restrict__ dst) {
    const int row = blockIdx.x, plane = blockIdx.y;
    const int64_t f = blockIdx.z;
    PlaneGeo g = plane_geo(D, plane);
    const int nsub = D.full ? D.pel * D.pel : 1;
    if (g.h <= 0 || row >= nsub * g.h || row >= g.rows) return;
    const int64_t src_frame = D.src_frame_bytes / (int64_t)sizeof(T), frame = D.frame_bytes / (int64_t)sizeof(T);
    L0View<T> V{src + f * src_frame + g.src_off, g.src_stride, g.w, g.h, g.stride};
    T *out = dst + f * frame + g.out_off + (int64_t)row * g.stride;
    const int pmax = D.px_max;
    const int p = row / g.h, y = row % g.h;
    const bool subpel = D.pel >= 2 && D.gpu <= 1 && D.full && p >= 1 && p <= 3;
    for (int64_t x = threadIdx.x; x < g.stride; x += blockDim.x) {
        unsigned v = 0;
        if (p == 0) {
            if (g.w > 0) v = V.L(y, x);
        } else if (subpel && x < g.w) {
            const int xi = (int)x;
            if (D.scale_up == 0) {  // fill_bilinear_pel2, super_build.rs:179-224
                if (p == 1) v = V.h_val(y, xi);
                else if (p == 2) v = y == 0 ? V.L(0, xi) : avg8(V.L(y, xi), V.flat((int64_t)(y + 1) * g.stride + xi));
                else v = y == 0 ? V.flat(1 + xi) : avg8(V.L(y, xi), V.flat((int64_t)(y + 1) * g.stride + 1 + xi));
            } else if (D.scale_up == 2) {  // fill_bicubic_pel2, super_build.rs:95-135
                auto row_h = [&](int yy) { return [&, yy](int xx) { return V.L(yy, xx); }; };
                auto colv = [&](int xx) { return [&, xx](int yy) { return V.L(yy, xx); }; };
                if (p == 1) v = half_tap(row_h(y), xi, g.w, pmax);
                else if (p == 2) v = half_tap(colv(xi), y, g.h, pmax);
                else v = half_tap([&](int xx) { return half_tap(colv(xx), y, g.h, pmax); }, xi, g.w, pmax);
            }
        }
        out[x] = (T)v;
    }
}

// reduce_6tap + horizontal_6tap_inplace, super_build.rs:254-357. One CTA per output row:
// the vertical pass for the whole row goes to shared memory, then the horizontal pass.
// Each output row receives src_w bytes: dst_w filtered values followed by the
// vertical-only intermediates of the remaining columns (the reference copies the whole
// intermediate row, :302-306), then zeros up to the pitch.
template <typename T>
__global__ void __launch_bounds__(256) super_reduce_kernel(SuperDev D, T *__restrict__ dst, int lv) {
    extern __shared__ __align__(16) uint8_t inter_raw[];
    T *inter = reinterpret_cast<T *>(inter_raw);
    const unsigned pmax = (unsigned)D.px_max;
    const int dy = blockIdx.x, plane = blockIdx.y;
    const int64_t f = blockIdx.z;
    PlaneGeo g = plane_geo(D, plane);
    const bool c = plane > 0;
    const int src_w = c ? D.lw[lv] / 2 : D.lw[lv], src_h = c ? D.lh[lv] / 2 : D.lh[lv];
    const int dst_w = c ? D.lw[lv + 1] / 2 : D.lw[lv + 1], dst_h = c ? D.lh[lv + 1] / 2 : D.lh[lv + 1];
    if (dy >= dst_h) return;
    const int64_t src_row0 = c ? D.row_c[lv] : D.row_y[lv];
    const int64_t drow = (c ? D.row_c[lv + 1] : D.row_y[lv + 1]) + dy;
    if (drow >= g.rows) return;
    T *base = dst + f * (D.frame_bytes / (int64_t)sizeof(T)) + g.out_off;
    T *out = base + drow * g.stride;
    const int64_t plane_len = g.rows * g.stride;
    const bool active = D.scale_down == 4 && dst_w > 0 && src_w > 0 && src_h > 0;
    if (!active) {
        for (int64_t x = threadIdx.x; x < g.stride; x += blockDim.x) out[x] = 0;
        return;
    }
    auto sample = [&](int64_t yy, int64_t xx) -> unsigned {
        int64_t i = (src_row0 + yy) * g.stride + xx;
        return i < plane_len ? base[i] : 0u;
    };
    const int sy = dy * 2;
    const bool use_edge = dy == 0 || dy + 1 == dst_h || sy - 2 < 0 || sy + 3 >= src_h;
    for (int x = threadIdx.x; x < src_w; x += blockDim.x) {
        unsigned v;
        if (use_edge) {
            int y0 = sy < src_h - 1 ? sy : src_h - 1, y1 = sy + 1 < src_h - 1 ? sy + 1 : src_h - 1;
            v = avg8(sample(y0, x), sample(y1, x));
        } else {
            int st = sy - 2;
            unsigned s = sample(st, x) + sample(st + 5, x) + 5u * (sample(st + 1, x) + sample(st + 4, x)) +
                         10u * (sample(st + 2, x) + sample(st + 3, x)) + 16u;
            v = s >> 5;
            v = v < pmax ? v : pmax;
        }
        inter[x] = (T)v;
    }
    __syncthreads();
    auto get = [&](int i, unsigned dflt) -> unsigned { return i < src_w ? inter[i] : dflt; };
    for (int64_t x = threadIdx.x; x < g.stride; x += blockDim.x) {
        unsigned v = 0;
        const int i = (int)x;
        if (x < dst_w) {
            if (dst_w <= 2) {
                unsigned a = get(2 * i, 0);
                v = avg8(a, get(2 * i + 1, a));
            } else if (i == 0 || i == dst_w - 1) {
                unsigned a = i == 0 ? inter[0] : get(2 * i, 0);
                v = avg8(a, get(2 * i + 1, a));
            } else {
                unsigned left = i == 1 ? avg8(inter[0], get(1, inter[0])) : get(2 * i - 2, 0);
                unsigned pk = get(2 * i + 3, inter[src_w - 1]);
                unsigned s = left + pk + 10u * (get(2 * i, 0) + get(2 * i + 1, 0)) + 5u * (get(2 * i - 1, 0) + get(2 * i + 2, 0)) + 16u;
                v = s >> 5;
                v = v < pmax ? v : pmax;
            }
        } else if (x < src_w) {
            v = inter[x];
        }
        out[x] = (T)v;
    }
}


// ---- 8-bit fast paths: rows processed in 16-byte (level 0) and 4-byte (reduction) words. Used
// when every row of the source and super frames starts on a 16-byte boundary; the kernels
// above serve every other geometry and the uint16 format. Both give the same bytes.

// rounded-up byte average of four packed bytes (avg_epu8, super_build.rs:250-253)
__device__ __forceinline__ uint32_t avgu4(uint32_t a, uint32_t b) { return (a | b) - (((a ^ b) >> 1) & 0x7F7F7F7Fu); }
__device__ __forceinline__ uint4 avg16(uint4 a, uint4 b) {
    return make_uint4(avgu4(a.x, b.x), avgu4(a.y, b.y), avgu4(a.z, b.z), avgu4(a.w, b.w));
}
// bytes 1..16 of (a, next byte)
__device__ __forceinline__ uint4 shift1(uint4 a, uint32_t next) {
    return make_uint4(__funnelshift_r(a.x, a.y, 8), __funnelshift_r(a.y, a.z, 8), __funnelshift_r(a.z, a.w, 8),
                      __funnelshift_r(a.w, next, 8));
}

// 16 bytes of sub-plane p of row y from x0 on, by the closed forms of super_level0_kernel
// (out of line: only the chunks at the right edge and in the last row take it).
// subpel: bilinear sub-pixel planes are filled (pel >= 2, gpu <= 1, full, scale.up 0).
__device__ __noinline__ uint4 level0_edge_chunk(bool subpel, const uint8_t *s0, int64_t sst, int w, int h, int64_t S,
                                                int y, int x0, int p) {
    const L0View<uint8_t> V{s0, sst, w, h, S};
    const PlaneGeo g{w, h, S, 0, 0, sst, 0};
    uint32_t wd0 = 0, wd1 = 0, wd2 = 0, wd3 = 0;
    for (int q = 0; q < 16; q++) {
        const int x = x0 + q;
        unsigned v = 0;
        if (p == 0) {
            if (g.w > 0) v = V.L(y, x);
        } else if (subpel && p <= 3 && x < g.w) {
            if (p == 1) v = V.h_val(y, x);
            else if (p == 2) v = y == 0 ? V.L(0, x) : avg8(V.L(y, x), V.flat((int64_t)(y + 1) * S + x));
            else v = y == 0 ? V.flat(1 + x) : avg8(V.L(y, x), V.flat((int64_t)(y + 1) * S + 1 + x));
        }
        const uint32_t b = (v & 0xFFu) << (8 * (q & 3));
        if (q < 4) wd0 |= b;
        else if (q < 8) wd1 |= b;
        else if (q < 12) wd2 |= b;
        else wd3 |= b;
    }
    return make_uint4(wd0, wd1, wd2, wd3);
}

// The level-0 region (copy + edge extension, super_build.rs:45-67; bilinear pel-2 planes,
// :179-224; zero sub-planes otherwise) of one 16-byte chunk of one row, every sub-plane of it.
// EDGE: the chunks reaching past the row's last sample (x0 + 16 > w) and those of the last row, by
// the scalar kernel's closed forms; otherwise the other chunks, in 16-byte words.
template <bool EDGE>
__device__ __forceinline__ void level0_chunk(const SuperDev &D, const uint8_t *__restrict__ src,
                                             uint8_t *__restrict__ dst, int plane, int64_t f, int y, int x0) {
    const PlaneGeo g = plane_geo(D, plane);
    const int S = (int)g.stride, w = g.w, h = g.h;
    const int nsub = D.full ? D.pel * D.pel : 1;
    const bool bil = D.pel >= 2 && D.gpu <= 1 && D.full && D.scale_up == 0;
    const uint8_t *s0 = src + f * D.src_frame_bytes + g.src_off;
    const int sst = (int)g.src_stride;
    uint8_t *o = dst + f * D.frame_bytes + g.out_off + (int64_t)y * S + x0;
    const int64_t pstep = (int64_t)h * S;  // one sub-plane further down
    const uint4 zero = make_uint4(0, 0, 0, 0);
    // sub-planes whose row y exists in the buffer (a super frame can have fewer rows than the
    // level-0 region, e.g. full:false, super_opts.rs:77-95)
    int np = 0;
    while (np < nsub && (int64_t)np * h + y < g.rows) np++;
    if (np == 0) return;
    if (!EDGE) {
        if (x0 + 16 > w || y + 1 >= h) return;  // the edge kernel's
        const uint8_t *r0 = s0 + (int64_t)y * sst + x0;
        const uint4 A = *reinterpret_cast<const uint4 *>(r0);
        *reinterpret_cast<uint4 *>(o) = A;
        if (nsub > 1) {
            uint4 p1 = zero, p2 = zero, p3 = zero;
            if (bil) {
                // the byte after the chunk in the super frame's flat memory (fill_bilinear_pel2 reads
                // it): the next sample; at the row's end the edge-extended padding (pitch > w) or the
                // next row's first sample (pitch == w)
                const bool last = x0 + 16 == w;
                const uint32_t nextA = !last ? r0[16] : (S > w ? (A.w >> 24) : r0[sst - x0]);
                const uint4 As = shift1(A, nextA);
                p1 = avg16(A, As);
                if (y == 0) {  // the v and hv planes' first rows are copies (copy_row, :205, :223)
                    p2 = A;
                    p3 = As;
                } else {
                    const uint8_t *r1 = r0 + sst;
                    const uint4 B = *reinterpret_cast<const uint4 *>(r1);
                    p2 = avg16(A, B);
                    // the byte after row y+1's chunk; past the last source row (pitch == w) it is the
                    // h plane's first byte, avg(L(0,0), L(0,1))
                    const uint32_t nextB = !last ? r1[16]
                                         : (S > w ? (B.w >> 24)
                                                  : (y + 2 < h ? r1[sst - x0] : avg8(s0[0], s0[w > 1 ? 1 : 0])));
                    p3 = avg16(A, shift1(B, nextB));
                }
            }
            if (np > 1) *reinterpret_cast<uint4 *>(o + pstep) = p1;
            if (np > 2) *reinterpret_cast<uint4 *>(o + 2 * pstep) = p2;
            if (np > 3) *reinterpret_cast<uint4 *>(o + 3 * pstep) = p3;
            for (int p = 4; p < np; p++) *reinterpret_cast<uint4 *>(o + p * pstep) = zero;
        }
        return;
    }
    const bool subpel = D.pel >= 2 && D.gpu <= 1 && D.full && D.scale_up == 0;
    for (int p = 0; p < np; p++)
        *reinterpret_cast<uint4 *>(o + p * pstep) = level0_edge_chunk(subpel, s0, g.src_stride, w, h, g.stride, y, x0, p);
}

// Every chunk of `nplanes` planes from plane0 on (luma, or both chroma planes) of every frame: a
// grid of resident CTAs strides over the items (frame, plane, row, chunk), so CTAs are few and
// each thread streams many chunks.
__global__ void __launch_bounds__(256, 4) super_level0_vec_kernel(SuperDev D, const uint8_t *__restrict__ src,
                                                               uint8_t *__restrict__ dst, int plane0, int nplanes,
                                                               int h, int chunks, uint32_t nitems) {
    for (uint32_t it = blockIdx.x * blockDim.x + threadIdx.x; it < nitems; it += gridDim.x * blockDim.x) {
        const uint32_t c = it % (uint32_t)chunks, r = it / (uint32_t)chunks;
        const uint32_t y = r % (uint32_t)h, fp = r / (uint32_t)h;
        level0_chunk<false>(D, src, dst, plane0 + (int)(fp % (uint32_t)nplanes), fp / (uint32_t)nplanes, (int)y,
                            (int)c * 16);
    }
}

// The edge chunks: per frame and plane, chunks [ce, chunks) of rows 0 .. h-2 (those reaching past
// the row's last sample), then the whole last row (ce = the chunks the vector kernel takes).
__global__ void __launch_bounds__(128) super_level0_edge_kernel(SuperDev D, const uint8_t *__restrict__ src,
                                                                uint8_t *__restrict__ dst, int plane0, int nplanes, int h,
                                                                int chunks, int ce, uint32_t nitems) {
    const uint32_t ne = (uint32_t)(chunks - ce), per = (uint32_t)(h - 1) * ne + (uint32_t)chunks;
    for (uint32_t it = blockIdx.x * blockDim.x + threadIdx.x; it < nitems; it += gridDim.x * blockDim.x) {
        const uint32_t e = it % per, fp = it / per;
        int y, c;
        if (e < (uint32_t)(h - 1) * ne) {
            y = (int)(e / ne);
            c = ce + (int)(e % ne);
        } else {
            y = h - 1;
            c = (int)(e - (uint32_t)(h - 1) * ne);
        }
        level0_chunk<true>(D, src, dst, plane0 + (int)(fp % (uint32_t)nplanes), fp / (uint32_t)nplanes, y, c * 16);
    }
}

// reduce_6tap + horizontal_6tap_inplace (super_build.rs:254-357) in 32-bit words. Each output
// row receives src_w bytes (dst_w filtered values, then the vertical-only intermediates,
// :302-306) and zeros up to the pitch.
// Bytes k1 and k2 (k2 - k1 <= 3) of the little-endian byte string W[0..3] that starts 4 bytes
// before the output word's first source byte, as the two low bytes of a halfword pair.
template <int K1, int K2>
__device__ __forceinline__ uint32_t pair_bytes(const uint32_t (&W)[4]) {
    constexpr int j = (K1 + 4) / 4, i1 = K1 + 4 - 4 * j, i2 = K2 + 4 - 4 * j;
    static_assert(j >= 0 && j + 1 < 4 && i2 < 8, "bytes within two neighbouring words");
    return __byte_perm(W[j], W[j + 1], (unsigned)(i1 | (i1 << 4) | (i2 << 8) | (i2 << 12))) & 0x00FF00FFu;
}
// horizontal_6tap_inplace's interior formula (:332-345) for outputs 2q and 2q + 1 of a word, in
// halfword lanes: output j = p[2j-2] + p[2j+3] + 10 (p[2j] + p[2j+1]) + 5 (p[2j-1] + p[2j+2]), + 16 >> 5.
template <int Q>
__device__ __forceinline__ uint32_t h6tap_pair(const uint32_t (&W)[4]) {
    constexpr int m = 4 * Q;  // source byte offset of the pair's first output, relative to 8 * word
    const uint32_t s = pair_bytes<m - 2, m>(W) + pair_bytes<m + 3, m + 5>(W) +
                       10u * (pair_bytes<m, m + 2>(W) + pair_bytes<m + 1, m + 3>(W)) +
                       5u * (pair_bytes<m - 1, m + 1>(W) + pair_bytes<m + 2, m + 4>(W)) + 0x00100010u;
    return (s >> 5) & 0x00FF00FFu;  // each lane <= 255: the weights sum to 32
}

// n / d for 0 <= n, 1 <= d with n * d < 2^32 by one high multiply: with m = ceil(2^32 / d) the
// error n (m d - 2^32) / 2^32 < 1 never carries past the next multiple of d (the band kernel's
// loop indices: n < 16 rows x 8192 words, d <= 8192).
struct FastDiv {
    uint32_t m;
    int d;
    __device__ __forceinline__ explicit FastDiv(int d_) : m(d_ > 1 ? 0xFFFFFFFFu / (uint32_t)d_ + 1u : 0u), d(d_) {}
    __device__ __forceinline__ int div(int n) const { return d > 1 ? (int)__umulhi((uint32_t)n, m) : n; }
};

// 16 bytes global -> shared without a register round trip (cp.async); completed by cp_async_wait.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(smem)), "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Output rows [r0, r0 + nr) of level lv + 1 of one plane of one frame, from level lv. The source
// rows the band reads (2 nr + 4 at most) go to shared memory in one burst of 16-byte
// asynchronous copies (every load of the band in flight at once), then the vertical 6-tap runs
// over (output row, 16-byte column chunk) pairs into the intermediate rows (bytes in halfword
// lanes), then the horizontal 6-tap, 4 output bytes per 32-bit store. Called by the whole CTA;
// `inter` holds nr intermediate rows, `in_sm` the staged source rows.
// lv0_src (level 0 only, nullable): read level 0's full-pel rows from the source frames instead of the
// super frames (the same bytes below the level's width; the rest is never used).
__device__ __forceinline__ void reduce_band(const SuperDev &D, uint8_t *__restrict__ dst, uint8_t *inter_all,
                                            uint8_t *in_sm, int plane, int64_t f, int lv, int r0, int nr,
                                            const uint8_t *__restrict__ lv0_src = nullptr) {
    const PlaneGeo g = plane_geo(D, plane);
    const bool c = plane > 0;
    const int S = (int)g.stride, SW = S >> 2;
    uint8_t *base = dst + f * D.frame_bytes + g.out_off;
    const int rows = (int)g.rows;
    const int src_w = c ? D.lw[lv] / 2 : D.lw[lv], src_h = c ? D.lh[lv] / 2 : D.lh[lv];
    const int dst_w = c ? D.lw[lv + 1] / 2 : D.lw[lv + 1], dst_h = c ? D.lh[lv + 1] / 2 : D.lh[lv + 1];
    const int srow0 = (int)(c ? D.row_c[lv] : D.row_y[lv]);
    const int drow0 = (int)(c ? D.row_c[lv + 1] : D.row_y[lv + 1]);
    const bool active = D.scale_down == 4 && dst_w > 0 && src_w > 0 && src_h > 0;
    const int iw = (src_w + 3) >> 2;        // intermediate words per row
    const int iq = (iw + 3) >> 2, ist = 4 * iq;  // 16-byte chunks per row; shared-memory row stride (words)
    if (active) {
        const uint4 z4 = make_uint4(0, 0, 0, 0);
        // source rows y_lo .. y_hi (the pitch is a multiple of 16, so a chunk stays inside its row;
        // rows past the buffer read as zeros)
        const int y_lo = max(2 * r0 - 2, 0), y_hi = min(2 * (r0 + nr - 1) + 3, src_h - 1);
        const uint4 *col = reinterpret_cast<const uint4 *>(
            lv0_src ? lv0_src + f * D.src_frame_bytes + g.src_off : base + (int64_t)srow0 * S);
        const int SQ = (int)((lv0_src ? g.src_stride : (int64_t)S) >> 4);
        const int have = lv0_src ? src_h : rows - srow0;  // source frames hold every level-0 row
        uint4 *in4 = reinterpret_cast<uint4 *>(in_sm);
        const FastDiv div_iq(iq);
        for (int t = threadIdx.x; t < (y_hi - y_lo + 1) * iq; t += blockDim.x) {
            const int rr = div_iq.div(t), cq = t - rr * iq, yy = y_lo + rr;
            if (yy < have) cp_async16(in4 + t, col + (int64_t)yy * SQ + cq);
            else in4[t] = z4;
        }
        cp_async_wait();
        __syncthreads();
        const uint32_t m = 0x00FF00FFu;
        auto vert = [&](uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t a4, uint32_t a5) -> uint32_t {
            const uint32_t e = (a0 & m) + (a5 & m) + 5u * ((a1 & m) + (a4 & m)) + 10u * ((a2 & m) + (a3 & m)) +
                               0x00100010u;
            const uint32_t od = ((a0 >> 8) & m) + ((a5 >> 8) & m) + 5u * (((a1 >> 8) & m) + ((a4 >> 8) & m)) +
                                10u * (((a2 >> 8) & m) + ((a3 >> 8) & m)) + 0x00100010u;
            return ((e >> 5) & m) | (((od >> 5) & m) << 8);  // each lane <= 255: weights sum to 32
        };
        for (int t = threadIdx.x; t < nr * iq; t += blockDim.x) {
            const int r = div_iq.div(t), cq = t - r * iq;
            auto row = [&](int yy) -> uint4 { return in4[(yy - y_lo) * iq + cq]; };
            const int dy = r0 + r, sy = 2 * dy;
            uint4 v;
            if (dy == 0 || dy + 1 == dst_h || sy - 2 < 0 || sy + 3 >= src_h) {
                const uint4 p = row(min(sy, src_h - 1)), q = row(min(sy + 1, src_h - 1));
                v = make_uint4(avgu4(p.x, q.x), avgu4(p.y, q.y), avgu4(p.z, q.z), avgu4(p.w, q.w));
            } else {
                const uint4 a0 = row(sy - 2), a1 = row(sy - 1), a2 = row(sy), a3 = row(sy + 1), a4 = row(sy + 2),
                            a5 = row(sy + 3);
                v = make_uint4(vert(a0.x, a1.x, a2.x, a3.x, a4.x, a5.x), vert(a0.y, a1.y, a2.y, a3.y, a4.y, a5.y),
                               vert(a0.z, a1.z, a2.z, a3.z, a4.z, a5.z), vert(a0.w, a1.w, a2.w, a3.w, a4.w, a5.w));
            }
            reinterpret_cast<uint4 *>(inter_all)[t] = v;  // row r at r * ist words
        }
    }
    __syncthreads();
    const FastDiv div_sw(SW);
    for (int t = threadIdx.x; t < nr * SW; t += blockDim.x) {
        const int r = div_sw.div(t), xw = t - r * SW;
        const int dy = r0 + r;
        uint32_t word = 0;
        if (!active || 4 * xw >= src_w) {
            // past the row's src_w bytes: zeros
        } else if (4 * xw >= dst_w && 4 * xw + 4 <= src_w) {
            word = reinterpret_cast<const uint32_t *>(inter_all)[r * ist + xw];  // vertical-only intermediates
        } else if (xw >= 1 && 4 * xw + 5 <= dst_w && 8 * xw + 9 < src_w) {
            // four interior outputs: source bytes 8xw-2 .. 8xw+9 of the row, in halfword lanes
            const uint32_t *in32 = reinterpret_cast<const uint32_t *>(inter_all) + r * ist + 2 * xw - 1;
            const uint32_t W[4] = {in32[0], in32[1], in32[2], in32[3]};
            word = __byte_perm(h6tap_pair<0>(W), h6tap_pair<1>(W), 0x6420);
        } else {
            const uint8_t *in = inter_all + r * ist * 4;
            auto get = [&](int i, unsigned dflt) -> unsigned { return i < src_w ? in[i] : dflt; };
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int i = xw * 4 + q;
                unsigned v = 0;
                if (i < dst_w) {
                    if (dst_w <= 2) {
                        const unsigned a = get(2 * i, 0);
                        v = avg8(a, get(2 * i + 1, a));
                    } else if (i == 0 || i == dst_w - 1) {
                        const unsigned a = i == 0 ? in[0] : get(2 * i, 0);
                        v = avg8(a, get(2 * i + 1, a));
                    } else {
                        const unsigned left = i == 1 ? avg8(in[0], get(1, in[0])) : get(2 * i - 2, 0);
                        const unsigned pk = get(2 * i + 3, in[src_w - 1]);
                        const unsigned sm = left + pk + 10u * (get(2 * i, 0) + get(2 * i + 1, 0)) +
                                            5u * (get(2 * i - 1, 0) + get(2 * i + 2, 0)) + 16u;
                        v = min(sm >> 5, 255u);
                    }
                } else if (i < src_w) {
                    v = in[i];
                }
                word |= v << (8 * q);
            }
        }
        if (drow0 + dy < rows) reinterpret_cast<uint32_t *>(base + (int64_t)(drow0 + dy) * S)[xw] = word;
    }
    __syncthreads();
}

// One pyramid level of every plane of every frame: a grid of resident CTAs strides over bands of
// `band` output rows (frame, plane, band), each CTA doing a band's vertical then horizontal pass.
__global__ void __launch_bounds__(256, 4) super_reduce_band_kernel(SuperDev D, uint8_t *__restrict__ dst, int lv, int band,
                                                                int nb_y, int nb_c, uint32_t nitems, int inter_bytes) {
    extern __shared__ __align__(16) uint8_t inter_all[];  // band intermediate rows, then the staged source rows
    const uint32_t per = (uint32_t)(nb_y + 2 * nb_c);
    for (uint32_t it = blockIdx.x; it < nitems; it += gridDim.x) {
        const uint32_t e = it % per;
        const int64_t f = it / per;
        int plane, b;
        if (e < (uint32_t)nb_y) { plane = 0; b = (int)e; }
        else { plane = 1 + (int)((e - nb_y) / (uint32_t)nb_c); b = (int)((e - nb_y) % (uint32_t)nb_c); }
        const int dst_h = plane ? D.lh[lv + 1] / 2 : D.lh[lv + 1];
        const int r0 = b * band;
        reduce_band(D, dst, inter_all, inter_all + inter_bytes, plane, f, lv, r0, min(band, dst_h - r0));
    }
}

// Level 0 and the level 0 -> 1 reduction in one launch. One CTA in kL01Split streams the level-0
// chunks of every plane, as super_level0_vec_kernel does: that work is bound by memory. The others
// reduce level-1 bands: that work is bound by instruction issue. They read level 0's full-pel rows from the
// source frames, so they need nothing the streaming CTAs write, and the two kinds of work share every
// SM instead of running one after the other.
constexpr uint32_t kL01Split = 2;  // measured: 1 in 2 CTAs streaming 1.34 ms, 1 in 4 2.47 ms
__global__ void __launch_bounds__(256, 4) super_level01_kernel(SuperDev D, const uint8_t *__restrict__ src,
                                                            uint8_t *__restrict__ dst, int chunks_y, int chunks_c,
                                                            uint32_t items_y, uint32_t items_c, int band, int nb_y,
                                                            int nb_c, uint32_t nbands, int inter_bytes) {
    extern __shared__ __align__(16) uint8_t inter_all[];
    // one CTA in kL01Split streams level 0, the others reduce bands (grid: a multiple of kL01Split)
    const uint32_t groups = gridDim.x / kL01Split, grp = blockIdx.x / kL01Split, role = blockIdx.x % kL01Split;
    if (role == 0) {
        const uint32_t cta = grp;
        const uint32_t hy = (uint32_t)D.height, hc = (uint32_t)(D.height / 2), step = groups * blockDim.x;
        for (uint32_t it = cta * blockDim.x + threadIdx.x; it < items_y; it += step) {
            const uint32_t c = it % (uint32_t)chunks_y, r = it / (uint32_t)chunks_y;
            level0_chunk<false>(D, src, dst, 0, r / hy, (int)(r % hy), (int)c * 16);
        }
        for (uint32_t it = cta * blockDim.x + threadIdx.x; it < items_c; it += step) {
            const uint32_t c = it % (uint32_t)chunks_c, r = it / (uint32_t)chunks_c;
            const uint32_t y = r % hc, fp = r / hc;
            level0_chunk<false>(D, src, dst, 1 + (int)(fp & 1u), fp >> 1, (int)y, (int)c * 16);
        }
        return;
    }
    const uint32_t cta = grp * (kL01Split - 1) + role - 1, nband_ctas = groups * (kL01Split - 1);
    const uint32_t per = (uint32_t)(nb_y + 2 * nb_c);
    for (uint32_t it = cta; it < nbands; it += nband_ctas) {
        const uint32_t e = it % per;
        const int64_t f = it / per;
        int plane, b;
        if (e < (uint32_t)nb_y) { plane = 0; b = (int)e; }
        else { plane = 1 + (int)((e - nb_y) / (uint32_t)nb_c); b = (int)((e - nb_y) % (uint32_t)nb_c); }
        const int dst_h = plane ? D.lh[1] / 2 : D.lh[1];
        const int r0 = b * band;
        reduce_band(D, dst, inter_all, inter_all + inter_bytes, plane, f, 0, r0, min(band, dst_h - r0), src);
    }
}

// Every row start of the source and super frames on a 16-byte boundary, 8-bit samples, and
// no bicubic planes: the fast paths apply.
bool vec_ok(const SuperDev &D, const void *src, const void *dst, int nframes) {
    auto a16 = [](int64_t v) { return (v & 15) == 0; };
    if ((int64_t)7 * ((D.width + 15) & ~15) > kBandSmemMax) return false;  // a band of one row must fit
    return D.px_bytes == 1 && D.scale_up != 2 && D.width >= 2 && (((uintptr_t)src | (uintptr_t)dst) & 15) == 0 &&
           a16(D.y_stride) && a16(D.c_stride) && a16(D.y_len) && a16(D.c_len) && a16(D.frame_bytes) &&
           a16(D.src_y_stride) && a16(D.src_c_stride) && a16(D.src_y_len) && a16(D.src_c_len) &&
           a16(D.src_frame_bytes) && D.y_rows * D.y_stride < (1ll << 31) && D.c_stride >= 4 &&
           (int64_t)nframes * D.height * (D.y_stride / 16) < (1ll << 31);
}
}  // namespace

namespace {
template <typename T>
int launch_super_t(const SuperDev &D, const T *src, T *dst, int nframes, cudaStream_t stream) {
    const int nsub = D.full ? D.pel * D.pel : 1;
    dim3 g0((unsigned)(nsub * D.height), 3, (unsigned)nframes);
    super_level0_kernel<T><<<g0, 256, 0, stream>>>(D, src, dst);
    int n = 1;
    for (int lv = 0; lv + 1 < D.levels; lv++) {
        int rows = D.lh[lv + 1];
        if (rows <= 0) continue;
        size_t smem = (size_t)(D.lw[lv] > 0 ? D.lw[lv] : 1) * sizeof(T);
        dim3 g((unsigned)rows, 3, (unsigned)nframes);
        super_reduce_kernel<T><<<g, 256, smem, stream>>>(D, dst, lv);
        n++;
    }
    return n;
}
}  // namespace

// The fast paths: level 0 in two launches each (luma, then both chroma planes; the chunks inside
// the rows, then the edge chunks), then one launch per pyramid level over bands of rows of every
// plane and frame.
// A level's band height: band rows of intermediates + 2 band + 4 staged source rows in about 54 KB,
// so four 256-thread CTAs fit an SM.
int band_rows(int row_bytes) { return std::max(1, std::min(16, ((54 << 10) / std::max(row_bytes, 1) - 4) / 3)); }

int launch_super_vec(const SuperDev &D, const uint8_t *src, uint8_t *dst, int nframes, int sms, cudaStream_t stream) {
    int n = 0;
    // level 0 and level 1 together (super_level01_kernel) when there is a level 1 of both planes and
    // the super frames hold every level-0 row (the source then stands in for them; a `full:false`
    // frame is shorter, and the rows it lacks read as zeros)
    const bool fused = D.levels > 1 && D.lh[1] / 2 > 0 && D.height / 2 > 0 && D.row_y[0] + D.lh[0] <= D.y_rows &&
                       D.row_c[0] + D.lh[0] / 2 <= D.c_rows;
    if (fused) {
        const int chunks_y = (int)(D.y_stride / 16), chunks_c = (int)(D.c_stride / 16);
        const uint32_t items_y = (uint32_t)((int64_t)nframes * D.height * chunks_y);
        const uint32_t items_c = (uint32_t)((int64_t)nframes * 2 * (D.height / 2) * chunks_c);
        const int row_bytes = (D.lw[0] + 15) & ~15, band = band_rows(row_bytes);
        const int nb_y = (D.lh[1] + band - 1) / band, nb_c = (D.lh[1] / 2 + band - 1) / band;
        const uint32_t nbands = (uint32_t)((int64_t)nframes * (nb_y + 2 * nb_c));
        super_level01_kernel<<<sms * 4, 256, (size_t)(3 * band + 4) * row_bytes, stream>>>(
            D, src, dst, chunks_y, chunks_c, items_y, items_c, band, nb_y, nb_c, nbands, band * row_bytes);
        n++;
    }
    for (int pl = 0; pl < 2; pl++) {
        const int64_t S = pl ? D.c_stride : D.y_stride;
        const int h = pl ? D.height / 2 : D.height;
        if (h <= 0) continue;
        const int nplanes = pl ? 2 : 1, chunks = (int)(S / 16);
        if (!fused) {
            const uint32_t nitems = (uint32_t)((int64_t)nframes * nplanes * h * chunks);
            const int grid = (int)std::min<int64_t>((nitems + 255) / 256, (int64_t)sms * 4);
            super_level0_vec_kernel<<<grid, 256, 0, stream>>>(D, src, dst, pl ? 1 : 0, nplanes, h, chunks, nitems);
            n++;
        }
        const int w = pl ? D.width / 2 : D.width;
        const int ce = std::min(w / 16, chunks);  // chunks with x0 + 16 <= w: the vector kernel's
        const uint32_t nedge = (uint32_t)((int64_t)nframes * nplanes * ((int64_t)(h - 1) * (chunks - ce) + chunks));
        super_level0_edge_kernel<<<(int)std::min<int64_t>((nedge + 127) / 128, (int64_t)sms * 8), 128, 0, stream>>>(
            D, src, dst, pl ? 1 : 0, nplanes, h, chunks, ce, nedge);
        n++;
    }
    for (int lv = fused ? 1 : 0; lv + 1 < D.levels; lv++) {
        const int dh_y = D.lh[lv + 1], dh_c = D.lh[lv + 1] / 2;
        if (dh_y <= 0) continue;
        const int row_bytes = (D.lw[lv] + 15) & ~15;  // the level's widest row (luma), 16-byte rows
        const int band = band_rows(row_bytes);
        const int nb_y = (dh_y + band - 1) / band, nb_c = (dh_c + band - 1) / band;
        const uint32_t nitems = (uint32_t)((int64_t)nframes * (nb_y + 2 * nb_c));
        const int grid = (int)std::min<int64_t>(nitems, (int64_t)sms * 4);
        const size_t smem = (size_t)(3 * band + 4) * row_bytes;
        super_reduce_band_kernel<<<grid, 256, smem, stream>>>(D, dst, lv, band, nb_y, nb_c, nitems, band * row_bytes);
        n++;
    }
    return n;
}

cudaError_t launch_super(const SuperDev &D, const uint8_t *src, uint8_t *dst, int nframes, cudaStream_t stream,
                         int *launches) {
    if (nframes <= 0) return cudaSuccess;
    static int sms = [] {
        int dev = 0, v = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            return 148;
        return v;
    }();
    if (vec_ok(D, src, dst, nframes)) {
        static const cudaError_t attr = [] {
            cudaError_t e = cudaFuncSetAttribute(super_reduce_band_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)kBandSmemMax);
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(super_level01_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kBandSmemMax);
            return e;
        }();
        if (attr != cudaSuccess) return attr;
        const int n = launch_super_vec(D, src, dst, nframes, sms, stream);
        if (launches) *launches += n;
        return cudaGetLastError();
    }
    const int n = D.px_bytes == 2
                      ? launch_super_t(D, reinterpret_cast<const uint16_t *>(src), reinterpret_cast<uint16_t *>(dst),
                                       nframes, stream)
                      : launch_super_t(D, src, dst, nframes, stream);
    if (launches) *launches += n;
    return cudaGetLastError();
}

bool make_super_dev(const SuperOpts &so, const SuperLayout &L, int64_t src_y_stride, int64_t src_c_stride,
                    SuperDev &D) {
    if (so.levels > kMaxLevels || so.levels < 0) return false;
    D.width = so.width; D.height = so.height; D.pel = so.pel; D.levels = so.levels; D.full = so.full;
    D.gpu = so.gpu; D.scale_up = so.scale_up; D.scale_down = so.scale_down;
    D.y_stride = L.y_stride; D.c_stride = L.c_stride;
    D.y_rows = L.super_h; D.c_rows = L.super_h / 2;
    D.y_len = L.y_len; D.c_len = L.c_len; D.frame_bytes = L.frame_bytes;
    D.px_bytes = so.bits > 8 ? 2 : 1;
    D.px_max = so.bits > 8 ? (1 << so.bits) - 1 : 255;
    D.src_y_stride = src_y_stride; D.src_c_stride = src_c_stride;
    D.src_y_len = src_y_stride * so.height;
    D.src_c_len = src_c_stride * (so.height / 2);
    D.src_frame_bytes = (D.src_y_len + 2 * D.src_c_len) * D.px_bytes;
    int64_t ry = 0, rc = 0;
    for (int lv = 0; lv < kMaxLevels; lv++) {
        D.lw[lv] = reduce_dim(so.width, lv);
        D.lh[lv] = reduce_dim(so.height, lv);
        D.row_y[lv] = ry;
        D.row_c[lv] = rc;
        int64_t sub = (lv == 0 && so.full) ? (int64_t)so.pel * so.pel : 1;
        ry += (int64_t)D.lh[lv] * sub;
        rc += (int64_t)(D.lh[lv] / 2) * sub;
    }
    return true;
}

}  // namespace svpf
