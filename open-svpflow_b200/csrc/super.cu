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
#include <stdint.h>

#include "svpf_device.h"

namespace svpf {

namespace {

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

cudaError_t launch_super(const SuperDev &D, const uint8_t *src, uint8_t *dst, int nframes, cudaStream_t stream,
                         int *launches) {
    if (nframes <= 0) return cudaSuccess;
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
