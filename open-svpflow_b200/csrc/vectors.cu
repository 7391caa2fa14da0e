// vectors.cu -- the consumer side of the Analyse payload on the device: decode the vectors
// and build the motion-vector planes a frame interpolator reads, without leaving HBM.
//
// Follows crates/svpflow-core/src/metadata.rs: vector_data (:89-115, the vdata header),
// motion_grid / extended_grid (:211-244), decode_vectors / decode_region (:246-273, :455-481);
// and renderer.rs: vector_planes (:1680-1726), clamp_to_frame (:1728-1736), sample_index
// (:1870-1874), centered (:3237-3243), as SmoothFps calls them (svpflow2 core.rs:962-1001): the
// "previous" set falls back to the current one and vice versa.
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <thread>
#include <vector>
#include <string>

#include "../../include/svpflow_b200.h"
#include "handles.h"

namespace {

namespace cg = cooperative_groups;
constexpr int kNeutral = 1024, kMaxVector = 1023;

struct VecHdr {  // vector_data(), from the 16-int vdata header
    int32_t flags, bw, bh, marker, w, h, ox, oy, gw, gh;
};

bool read_vdata(const int32_t *v, VecHdr &h) {
    if (!v || v[0] != 0xA0) return false;  // VECTOR_MAGIC
    h.flags = v[1]; h.bw = v[2]; h.bh = v[3]; h.marker = v[4];
    h.w = v[7]; h.h = v[8]; h.ox = v[9]; h.oy = v[10]; h.gw = v[11]; h.gh = v[12];
    return true;
}
inline int extended_grid(int block, int overlap, int grid, int source) {
    const long long span = (long long)(block - overlap) * grid + overlap;
    return grid + (span < source ? 1 : 0);
}

struct PlaneJob {
    const uint8_t *payloads;
    int64_t payload_len;
    uint16_t *planes;     // per payload: mvx0 | mvy0 | mvx1 | mvy1, each mw x mh
    int *status;          // per payload: 0 ok, 1 the payload does not decode
    int32_t flags, gw, gh, mw, mh;
    int32_t bw, bh, step_x, step_y, frame_w, frame_h, raw;
};

__device__ __forceinline__ int rd32(const uint8_t *p, int64_t len, int64_t off, bool &ok) {
    if (off < 0 || off + 4 > len) { ok = false; return 0; }
    return *reinterpret_cast<const int *>(p + off);
}

__device__ __forceinline__ int clamp_to_frame(int value, int pos, int block, int frame) {
    if (value + pos < 0) return -pos;
    if (value + block + pos > frame) return frame - block - pos > 0 ? frame - block - pos : 0;
    return value;
}
__device__ __forceinline__ uint16_t centered(int v) {
    if (v > kMaxVector || v < -kMaxVector) return (uint16_t)kNeutral;
    return (uint16_t)(v + kNeutral);
}

// decode_vectors' checks on one payload (every thread reads the same few words): header, region
// markers, region lengths. On success, the byte offsets of the two sets' first vectors, the
// previous set falling back to the current one and vice versa.
__device__ __forceinline__ bool decode_regions(const uint8_t *p, int64_t len, int32_t flags, int64_t count,
                                               int64_t &off_prev, int64_t &off_cur) {
    const int64_t first = 0x40, second = first + 4 + count * 8;
    bool ok = true;
    const bool hdr = rd32(p, len, 0, ok) == 16 && rd32(p, len, 4, ok) == 0xA0 && rd32(p, len, 8, ok) == flags;
    const int marker = (int)(2 * count + 1);
    const bool has_prev = (flags & 1) != 0, has_cur = (flags & 2) != 0;
    if (has_prev && rd32(p, len, first, ok) != marker) ok = false;
    if (has_cur && rd32(p, len, second, ok) != marker) ok = false;
    if (has_prev && first + 4 + count * 8 > len) ok = false;
    if (has_cur && second + 4 + count * 8 > len) ok = false;
    off_prev = has_prev ? first + 4 : second + 4;
    off_cur = has_cur ? second + 4 : first + 4;
    return ok && hdr && (has_prev || has_cur);
}

// grid: (positions / 256, payloads)
__global__ void vector_planes_kernel(const PlaneJob J) {
    const int64_t f = blockIdx.y;
    const uint8_t *p = J.payloads + f * J.payload_len;
    const int64_t count = (int64_t)J.gw * J.gh;
    int64_t off_prev, off_cur;
    if (!decode_regions(p, J.payload_len, J.flags, count, off_prev, off_cur)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) J.status[f] = 1;
        return;
    }
    const int64_t n = (int64_t)J.mw * J.mh;
    uint16_t *out = J.planes + f * 4 * n;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % J.mw), y = (int)(i / J.mw);
        const int sx = x < J.gw - 1 ? x : (J.gw > 0 ? J.gw - 1 : 0), sy = y < J.gh - 1 ? y : (J.gh > 0 ? J.gh - 1 : 0);
        const int64_t si = (int64_t)sy * J.gw + sx;  // sample_index
        const int pos_x = x * J.step_x, pos_y = y * J.step_y;
        for (int which = 0; which < 2; which++) {
            int dx = 0, dy = 0;
            if (si < count) {
                const unsigned raw0 = *reinterpret_cast<const unsigned *>(p + (which ? off_cur : off_prev) + si * 8);
                dx = (int)(short)(raw0 >> 16);
                dy = (int)(short)(raw0 & 0xFFFF);
            }
            uint16_t ox, oy;
            if (dx > kMaxVector || dx < -kMaxVector || dy > kMaxVector || dy < -kMaxVector) {
                ox = oy = (uint16_t)kNeutral;
            } else {
                if (!J.raw) {
                    dx = clamp_to_frame(dx, pos_x, J.bw, J.frame_w);
                    dy = clamp_to_frame(dy, pos_y, J.bh, J.frame_h);
                }
                ox = centered(dx);
                oy = centered(dy);
            }
            out[(2 * which) * n + i] = ox;
            out[(2 * which + 1) * n + i] = oy;
        }
    }
}

// ---------------------------------------------------------------- mask planes
// SmoothFps' masks for one interpolated frame (svpflow2 core.rs:1154-1195, :1467-1499, :1605-1616):
// renderer.rs coverage_mask (:1738-1763) = splat_coverage (:2945-3062) + window_3x3 (:3064-3100) +
// finish_coverage (:3102-3134), and magnitude_mask (:1647-1678) with scale_magnitude (:3245-3260).
// The splat's weights are >= 0 when 0 <= overlap < block, so every partial sum is bounded by
// grid_w * grid_h * block area; the host admits only fields where that is <= 2^30, which makes the
// reference's saturating and wrapping adds plain adds and the atomic sums order-independent.
// TruncDiv (:3149-3184) divides exactly (truncating), so plain '/' restates it.

constexpr int kMagRuns = 512;  // the most runs of equal magnitude bytes a setting may have

struct MaskJob {
    const uint8_t *payloads;
    int64_t payload_len;
    uint8_t *masks;       // per payload: cover0 | cover1 | area0 | area1 | max(area0, area1), each mw x mh
    int32_t *sums;        // per payload: two (mw + 2) x (mh + 2) splat planes
    int *status;
    int32_t flags, gw, gh, mw, mh;
    int32_t bw, bh, xs, ys, denom, phase, area, sharp_is_one, mag_steps, mag_runs;
    double strength, area_scale, area_sharp;
    // mag_steps: the magnitude byte is the number of these scores at or below the vector's score
    uint32_t mag_thr[255];
    // mag_runs > 0 (any other setting): the byte of a score is mag_run_byte[i] for the last run i
    // with mag_run_start[i] <= score (mag_run_start[0] = 0)
    uint32_t mag_run_start[kMagRuns];
    uint8_t mag_run_byte[kMagRuns];
};

__device__ __forceinline__ bool mask_regions(const MaskJob &J, const uint8_t *p, int64_t &off_prev,
                                             int64_t &off_cur) {
    return decode_regions(p, J.payload_len, J.flags, (int64_t)J.gw * J.gh, off_prev, off_cur);
}

// grid: (vectors / 256, payloads, 2). z = 0: mask 0 splats the current set at 256 - phase;
// z = 1: mask 1 splats the previous set at phase (coverage_mask's opposite_set).
__global__ void mask_splat_kernel(const MaskJob J) {
    const int64_t f = blockIdx.y;
    const int which = blockIdx.z;
    const uint8_t *p = J.payloads + f * J.payload_len;
    int64_t off_prev, off_cur;
    if (!mask_regions(J, p, off_prev, off_cur)) return;
    const int64_t count = (int64_t)J.gw * J.gh;
    const int64_t stride = (int64_t)J.mw + 2;
    int32_t *acc = J.sums + (f * 2 + which) * stride * ((int64_t)J.mh + 2);
    const int64_t off = which ? off_prev : off_cur;
    const int t = which ? J.phase : 256 - J.phase;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < count; k += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(k % J.gw), y = (int)(k / J.gw);
        const unsigned raw0 = *reinterpret_cast<const unsigned *>(p + off + k * 8);
        const int vdx = (int)(short)(raw0 >> 16), vdy = (int)(short)(raw0 & 0xFFFF);
        const int sx = x * J.xs + (t * vdx) / J.denom;
        const int sy = y * J.ys + (t * vdy) / J.denom;
        // floor division (the reference biases negative numerators by 1 - step)
        const int left = (sx + ((1 - J.xs) & (sx >> 31))) / J.xs;
        const int top = (sy + ((1 - J.ys) & (sy >> 31))) / J.ys;
        const int right = left + 1, bottom = top + 1;
        const int next_x = right * J.xs;
        const int lw = next_x - sx, tw = J.ys * bottom - sy, rw = sx + J.bw - next_x, bwt = J.bh - tw;
        // the interior path and add_point's four conditions both reduce to: corners inside mw x mh
        const bool l_in = left >= 0 && left < J.mw, r_in = right >= 0 && right < J.mw;
        const bool t_in = top >= 0 && top < J.mh, b_in = bottom >= 0 && bottom < J.mh;
        if (t_in && l_in) atomicAdd(acc + (int64_t)top * stride + left, lw * tw);
        if (t_in && r_in) atomicAdd(acc + (int64_t)top * stride + right, tw * rw);
        if (b_in && r_in) atomicAdd(acc + (int64_t)bottom * stride + right, rw * bwt);
        if (b_in && l_in) atomicAdd(acc + (int64_t)bottom * stride + left, lw * bwt);
    }
}

__device__ __forceinline__ uint8_t coverage_byte(double v) {
    if (!isfinite(v)) return 0;
    const int i = __double2int_rz(v);  // saturating, as Rust's `as i32`
    return i >= 255 ? 255 : (uint8_t)(i & 0xFF);
}
__device__ __forceinline__ uint8_t clamp_u8(double v) {
    if (!isfinite(v) || v <= 0.0) return 0;
    if (v >= 255.0) return 255;
    return (uint8_t)__double2int_rz(v);
}

// grid: (points / 256, payloads): window_3x3 + finish_coverage for both masks, and both magnitude masks.
__global__ void mask_finish_kernel(const MaskJob J) {
    const int64_t f = blockIdx.y;
    const uint8_t *p = J.payloads + f * J.payload_len;
    int64_t off_prev, off_cur;
    if (!mask_regions(J, p, off_prev, off_cur)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) J.status[f] = 1;
        return;
    }
    __shared__ uint32_t thr[255];
    __shared__ uint32_t run_start[kMagRuns];
    __shared__ uint8_t run_byte[kMagRuns];
    if (J.mag_steps) {  // the whole block takes this branch or returned above
        for (int k = threadIdx.x; k < 255; k += blockDim.x) thr[k] = J.mag_thr[k];
        __syncthreads();
    } else if (J.mag_runs) {
        for (int k = threadIdx.x; k < J.mag_runs; k += blockDim.x) {
            run_start[k] = J.mag_run_start[k];
            run_byte[k] = J.mag_run_byte[k];
        }
        __syncthreads();
    }
    const int64_t n = (int64_t)J.mw * J.mh;
    const int64_t stride = (int64_t)J.mw + 2, plane = stride * ((int64_t)J.mh + 2);
    const int32_t *acc = J.sums + f * 2 * plane;
    uint8_t *out = J.masks + f * 5 * n;
    const double area_f = (double)J.area;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % J.mw), y = (int)(i / J.mw);
        const int x0 = x > 0 ? x - 1 : 0, y0 = y > 0 ? y - 1 : 0;
        for (int m = 0; m < 2; m++) {
            int s = 0;  // the 3x3 window around (x, y); rows / columns past the plane hold 0
            for (int yy = y0; yy <= y + 1; yy++)
                for (int xx = x0; xx <= x + 1; xx++) s += __ldg(acc + m * plane + (int64_t)yy * stride + xx);
            const int covered = s >> 3;
            const int remaining = J.area <= covered ? 0 : J.area - covered;
            out[m * n + i] = coverage_byte(__ddiv_rn(__dmul_rn(__dmul_rn((double)remaining, J.strength), 256.0), area_f));
        }
        // magnitude_mask's fill: columns past the grid repeat the row's last vector, rows past it
        // repeat the grid's bottom-left one
        int64_t si = -1;
        if (J.gw > 0 && J.gh > 0) si = y < J.gh ? (int64_t)y * J.gw + (x < J.gw ? x : J.gw - 1) : (int64_t)(J.gh - 1) * J.gw;
        uint8_t a[2] = {0, 0};
        if (si >= 0)
            for (int s = 0; s < 2; s++) {
                const unsigned raw1 = *reinterpret_cast<const unsigned *>(p + (s ? off_cur : off_prev) + si * 8 + 4);
                const unsigned score = raw1 & 0xFFFFFFu;
                if (J.mag_steps) {  // count the step scores <= score (they ascend)
                    int lo = 0, hi = 255;
                    while (lo < hi) {
                        const int mid = (lo + hi) >> 1;
                        if (thr[mid] <= score) lo = mid + 1;
                        else hi = mid;
                    }
                    a[s] = (uint8_t)lo;
                } else if (J.mag_runs) {  // the last run starting at or below score
                    int lo = 0, hi = J.mag_runs - 1;
                    while (lo < hi) {
                        const int mid = (lo + hi + 1) >> 1;
                        if (run_start[mid] <= score) lo = mid;
                        else hi = mid - 1;
                    }
                    a[s] = run_byte[lo];
                } else {
                    double v = __ddiv_rn(__dmul_rn(__dmul_rn(4.0, (double)score), J.area_scale), area_f);
                    if (!J.sharp_is_one) v = pow(v, J.area_sharp);
                    a[s] = clamp_u8(__dmul_rn(v, 255.0));
                }
            }
        out[2 * n + i] = a[0];
        out[3 * n + i] = a[1];
        out[4 * n + i] = a[0] > a[1] ? a[0] : a[1];
    }
}

// ---------------------------------------------------------------- scene class
// SmoothFps's scene class of a payload (svpflow2 core.rs:2079-2100): metadata.rs analyze_scene
// (:349-361) = luma_map (:275-297) + classify_scene (:299-347). luma_byte (:523-526) of
// (previous luma + current luma) / denom takes at most 511 inputs, so the host tabulates it with
// libm's pow (the reference's own) and the kernel only looks it up: the counts are integer.
struct SceneJob {
    const uint8_t *payloads;
    int64_t payload_len;
    int32_t *classes, *status;
    int32_t flags, gw, gh;
    int32_t blocks_pct, zero, m1, m2, scene;
    uint8_t luma[512];  // luma_byte of (a + b) / denom, a + b in 0..510
};

// grid: (kSceneCtas x payloads); a cluster of kSceneCtas CTAs reduces one payload: each CTA counts
// its share of the vectors into the four bins (warp shuffles), adds them into the lead CTA's shared
// counters through distributed shared memory, and the lead CTA derives the class after the
// cluster barrier.
constexpr int kSceneCtas = 8;
__global__ void __cluster_dims__(kSceneCtas, 1, 1) __launch_bounds__(256)
    scene_class_kernel(const __grid_constant__ SceneJob J) {
    __shared__ int cnt[4];  // considered, scene, m2, m1 (the lead CTA's are the payload's)
    cg::cluster_group cluster = cg::this_cluster();
    const unsigned rank = cluster.block_rank();
    const int64_t f = blockIdx.x / kSceneCtas;
    const uint8_t *p = J.payloads + f * J.payload_len;
    const int64_t count = (int64_t)J.gw * J.gh;
    // the same checks in every CTA of the cluster, so all of them return or none does
    bool ok = true;
    const bool hdr = rd32(p, J.payload_len, 0, ok) == 16 && rd32(p, J.payload_len, 4, ok) == 0xA0 &&
                     rd32(p, J.payload_len, 8, ok) == J.flags;
    int64_t off_prev = 0, off_cur = 0;
    const bool sets = (J.flags & 3) != 0;
    if (ok && hdr && sets) ok = decode_regions(p, J.payload_len, J.flags, count, off_prev, off_cur);
    if (!(ok && hdr)) {
        if (rank == 0 && threadIdx.x == 0) { J.status[f] = 1; J.classes[f] = -1; }
        return;
    }
    if (!sets) {  // no vector set: scene_class returns 3
        if (rank == 0 && threadIdx.x == 0) J.classes[f] = 3;
        return;
    }
    if (threadIdx.x < 4) cnt[threadIdx.x] = 0;
    cluster.sync();  // the lead CTA's counters are zero before anyone adds
    int c[4] = {0, 0, 0, 0};
    for (int64_t i = (int64_t)rank * blockDim.x + threadIdx.x; i < count; i += (int64_t)kSceneCtas * blockDim.x) {
        const unsigned lp = *reinterpret_cast<const unsigned *>(p + off_prev + i * 8 + 4) >> 24;
        const unsigned wc = *reinterpret_cast<const unsigned *>(p + off_cur + i * 8 + 4);
        const int l = max((int)J.luma[lp + (wc >> 24)], 1);
        const long long s255 = (long long)(wc & 0xFFFFFFu) * 255;
        const int score = (int)(s255 > INT32_MAX ? INT32_MAX : s255) / l;  // saturating_mul, then /
        if (score < J.zero) continue;
        c[0]++;
        if (score >= J.scene) c[1]++;
        else if (score >= J.m2) c[2]++;
        else if (score >= J.m1) c[3]++;
    }
    int *lead = cluster.map_shared_rank(cnt, 0);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        int v = c[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
        if ((threadIdx.x & 31) == 0 && v) atomicAdd(lead + k, v);
    }
    cluster.sync();  // every CTA's counts are in
    if (rank == 0 && threadIdx.x == 0) {
        const int required = (int)((unsigned)cnt[0] * (unsigned)J.blocks_pct) / 100;
        const int high = cnt[1] + cnt[2], mid = high + cnt[3];
        J.classes[f] = cnt[1] >= required ? 3 : (high >= required ? 2 : (mid >= required ? 1 : 0));
    }
}

// scale_magnitude (renderer.rs:3245-3260) on the host, with libm's pow as the reference
uint8_t magnitude_byte(uint32_t score, double scale, double sharp, int32_t area) {
    const double v = pow(4.0 * (double)score * scale / (double)area, sharp) * 255.0;
    if (!isfinite(v) || v <= 0.0) return 0;
    if (v >= 255.0) return 255;
    return (uint8_t)v;
}
// For sharp >= 1e-3 and scale >= 0 the byte is a non-decreasing step function of the 24-bit score
// (scores one apart differ by >= 2^-24 relative, so pow's sub-ulp error cannot reorder them): the
// smallest score reaching each byte 1..255 (2^24 = never) makes the device result libm's exactly.
bool magnitude_steps(double scale, double sharp, int32_t area, uint32_t thr[255]) {
    if (!(sharp >= 1e-3) || !isfinite(sharp) || !(scale >= 0.0) || !isfinite(scale) || area <= 0) return false;
    static std::mutex mu;
    static double c_scale = -1.0, c_sharp = -1.0;
    static int32_t c_area = -1;
    static uint32_t c_thr[255];
    std::lock_guard<std::mutex> lk(mu);
    if (scale != c_scale || sharp != c_sharp || area != c_area) {
        for (int k = 1; k <= 255; k++) {
            uint32_t lo = 0, hi = 1u << 24;  // first score in [lo, hi) whose byte reaches k; hi = none
            while (lo < hi) {
                const uint32_t mid = lo + ((hi - lo) >> 1);
                if (magnitude_byte(mid, scale, sharp, area) >= k) hi = mid;
                else lo = mid + 1;
            }
            c_thr[k - 1] = lo;
        }
        c_scale = scale; c_sharp = sharp; c_area = area;
    }
    memcpy(thr, c_thr, sizeof(c_thr));
    return true;
}

// Every other setting (sharpness below 1e-3 or not positive, negative or non-finite scale): libm's
// byte for each of the 2^24 scores, as runs of equal bytes (a handful for any setting: the byte is
// a monotone function of the score, or NaN-to-0 apart from score 0). False when there are more
// than kMagRuns runs; the kernel then calls CUDA's pow (bytes not guaranteed equal to libm's).
bool magnitude_runs(double scale, double sharp, int32_t area, uint32_t *start, uint8_t *byte, int32_t *nruns) {
    if (area <= 0) return false;
    static std::mutex mu;
    static double c_scale = 0.0, c_sharp = 0.0;
    static int32_t c_area = -1, c_n = 0;
    static uint32_t c_start[kMagRuns];
    static uint8_t c_byte[kMagRuns];
    std::lock_guard<std::mutex> lk(mu);
    const bool same = c_area == area && memcmp(&c_scale, &scale, sizeof(double)) == 0 &&
                      memcmp(&c_sharp, &sharp, sizeof(double)) == 0;
    if (!same) {
        constexpr uint32_t kScores = 1u << 24;
        const unsigned nt = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
        std::vector<std::vector<std::pair<uint32_t, uint8_t>>> part(nt);
        std::vector<std::thread> th;
        for (unsigned t = 0; t < nt; t++)
            th.emplace_back([&, t] {
                const uint32_t a = (uint32_t)((uint64_t)kScores * t / nt), b = (uint32_t)((uint64_t)kScores * (t + 1) / nt);
                int prev = -1;
                for (uint32_t sc = a; sc < b; sc++) {
                    const uint8_t v = magnitude_byte(sc, scale, sharp, area);
                    if (v != prev) {
                        part[t].push_back({sc, v});
                        prev = v;
                        if (part[t].size() > (size_t)kMagRuns) return;
                    }
                }
            });
        for (auto &x : th) x.join();
        int n = 0;
        bool ok = true;
        for (unsigned t = 0; t < nt && ok; t++)
            for (auto &r : part[t]) {
                if (n > 0 && c_byte[n - 1] == r.second) continue;  // a run that continues across threads
                if (n == kMagRuns || part[t].size() > (size_t)kMagRuns) { ok = false; break; }
                c_start[n] = r.first;
                c_byte[n] = r.second;
                n++;
            }
        c_scale = scale; c_sharp = sharp; c_area = area; c_n = ok ? n : 0;
    }
    if (c_n == 0) return false;
    memcpy(start, c_start, sizeof(uint32_t) * (size_t)c_n);
    memcpy(byte, c_byte, (size_t)c_n);
    *nruns = c_n;
    return true;
}

bool mask_job(const int32_t *vdata, MaskJob &J, std::string &err) {
    VecHdr h;
    if (!read_vdata(vdata, h)) {
        err = "not a vector header";
        return false;
    }
    J.flags = h.flags;
    J.gw = h.gw > 0 ? h.gw : 0;
    J.gh = h.gh > 0 ? h.gh : 0;
    J.mw = extended_grid(h.bw, h.ox, h.gw, h.w);
    J.mh = extended_grid(h.bh, h.oy, h.gh, h.h);
    if (J.mw < 0) J.mw = 0;
    if (J.mh < 0) J.mh = 0;
    J.bw = h.bw > 1 ? h.bw : 1;
    J.bh = h.bh > 1 ? h.bh : 1;
    if (h.ox < 0 || h.oy < 0 || h.ox >= J.bw || h.oy >= J.bh) {
        err = "overlap outside 0..block - 1";
        return false;
    }
    if ((int64_t)J.gw * J.gh * J.bw * J.bh > INT32_MAX / 2 || (int64_t)(J.mw + 2) * (J.mh + 2) > INT32_MAX) {
        err = "vector field too large for 32-bit coverage sums";
        return false;
    }
    J.xs = J.bw - h.ox;
    J.ys = J.bh - h.oy;
    J.denom = (int32_t)((uint32_t)(h.marker > 1 ? h.marker : 1) << 8);
    J.area = (int64_t)J.bw * J.bh > INT32_MAX ? INT32_MAX : J.bw * J.bh;
    return true;
}

}  // namespace

extern "C" {

int svpf_vector_grid(const int32_t *vdata, int32_t *motion_w, int32_t *motion_h) {
    VecHdr h;
    if (!read_vdata(vdata, h)) {
        svpf::set_last_error("not a vector header");
        return SVPF_EINVAL;
    }
    if (motion_w) *motion_w = extended_grid(h.bw, h.ox, h.gw, h.w);
    if (motion_h) *motion_h = extended_grid(h.bh, h.oy, h.gh, h.h);
    return SVPF_OK;
}

int svpf_vector_planes_device(const int32_t *vdata, const uint8_t *payloads_dev, size_t payload_len, int32_t npayloads,
                              int32_t frame_w, int32_t frame_h, int32_t raw, uint16_t *planes_dev, int32_t *status_dev,
                              void *stream) {
    if (int rc = svpf::require_device()) return rc;
    VecHdr h;
    if (!read_vdata(vdata, h)) {
        svpf::set_last_error("not a vector header");
        return SVPF_EINVAL;
    }
    if (npayloads <= 0) return SVPF_OK;
    if (!payloads_dev || !planes_dev || !status_dev || payload_len < 0x40 || npayloads > 65535) {
        svpf::set_last_error("bad buffers");
        return SVPF_EINVAL;
    }
    if ((payload_len & 3) || ((uintptr_t)payloads_dev & 3) || ((uintptr_t)planes_dev & 1)) {
        svpf::set_last_error("payloads must be 4-byte aligned");
        return SVPF_EINVAL;
    }
    PlaneJob J;
    J.payloads = payloads_dev;
    J.payload_len = (int64_t)payload_len;
    J.planes = planes_dev;
    J.status = status_dev;
    J.flags = h.flags;
    J.gw = h.gw > 0 ? h.gw : 0;
    J.gh = h.gh > 0 ? h.gh : 0;
    J.mw = extended_grid(h.bw, h.ox, h.gw, h.w);
    J.mh = extended_grid(h.bh, h.oy, h.gh, h.h);
    if (J.mw < 0) J.mw = 0;
    if (J.mh < 0) J.mh = 0;
    J.bw = h.bw > 1 ? h.bw : 1;   // block.width.max(1)
    J.bh = h.bh > 1 ? h.bh : 1;
    J.step_x = J.bw - h.ox;       // block_w - origin_x
    J.step_y = J.bh - h.oy;
    J.frame_w = frame_w;
    J.frame_h = frame_h;
    J.raw = raw != 0;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(status_dev, 0, sizeof(int32_t) * (size_t)npayloads, st);
    const int64_t n = (int64_t)J.mw * J.mh;
    if (e == cudaSuccess && n > 0) {
        dim3 grid((unsigned)((n + 255) / 256 < 65535 ? (n + 255) / 256 : 65535), (unsigned)npayloads);
        vector_planes_kernel<<<grid, 256, 0, st>>>(J);
        svpf::add_launches(1);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        svpf::set_last_error(std::string("vector planes: ") + cudaGetErrorString(e));
        return SVPF_ECUDA;
    }
    return SVPF_OK;
}

}  // extern "C"

extern "C" {

int64_t svpf_render_masks_scratch(const int32_t *vdata, int32_t npayloads) {
    MaskJob J;
    std::string err;
    if (npayloads < 0 || !mask_job(vdata, J, err)) {
        svpf::set_last_error(npayloads < 0 ? std::string("negative payload count") : err);
        return -1;
    }
    return (int64_t)npayloads * 2 * ((int64_t)J.mw + 2) * ((int64_t)J.mh + 2) * (int64_t)sizeof(int32_t);
}

int svpf_render_masks_device(const int32_t *vdata, const uint8_t *payloads_dev, size_t payload_len, int32_t npayloads,
                             int32_t phase, int32_t cover_percent, double area_scale, double area_sharp,
                             uint8_t *masks_dev, void *scratch_dev, int32_t *status_dev, void *stream) {
    if (int rc = svpf::require_device()) return rc;
    MaskJob J;
    std::string err;
    if (!mask_job(vdata, J, err)) {
        svpf::set_last_error(err);
        return SVPF_EINVAL;
    }
    if (phase < 0 || phase > 256 || cover_percent < 0) {
        svpf::set_last_error("phase must be in 0..256 and cover >= 0");
        return SVPF_EINVAL;
    }
    if (npayloads <= 0) return SVPF_OK;
    if (!payloads_dev || !masks_dev || !scratch_dev || !status_dev || payload_len < 0x40 || npayloads > 65535) {
        svpf::set_last_error("bad buffers");
        return SVPF_EINVAL;
    }
    if ((payload_len & 3) || ((uintptr_t)payloads_dev & 3) || ((uintptr_t)scratch_dev & 3)) {
        svpf::set_last_error("payloads and scratch must be 4-byte aligned");
        return SVPF_EINVAL;
    }
    J.payloads = payloads_dev;
    J.payload_len = (int64_t)payload_len;
    J.masks = masks_dev;
    J.sums = static_cast<int32_t *>(scratch_dev);
    J.status = status_dev;
    J.phase = phase;
    J.strength = (double)cover_percent / 100.0;
    J.area_scale = area_scale;
    J.area_sharp = area_sharp;
    J.sharp_is_one = area_sharp == 1.0;  // pow(x, 1) is x exactly, in libm and here
    J.mag_steps = magnitude_steps(area_scale, area_sharp, J.area, J.mag_thr) ? 1 : 0;
    J.mag_runs = 0;
    if (!J.mag_steps && !magnitude_runs(area_scale, area_sharp, J.area, J.mag_run_start, J.mag_run_byte, &J.mag_runs))
        J.mag_runs = 0;
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t n = (int64_t)J.mw * J.mh, count = (int64_t)J.gw * J.gh;
    const size_t sums = (size_t)npayloads * 2 * ((size_t)J.mw + 2) * ((size_t)J.mh + 2) * sizeof(int32_t);
    cudaError_t e = cudaMemsetAsync(status_dev, 0, sizeof(int32_t) * (size_t)npayloads, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(scratch_dev, 0, sums, st);
    if (e == cudaSuccess && count > 0 && n > 0 && J.denom != 0) {  // splat_coverage returns early on denom 0
        dim3 grid((unsigned)((count + 255) / 256 < 65535 ? (count + 255) / 256 : 65535), (unsigned)npayloads, 2);
        mask_splat_kernel<<<grid, 256, 0, st>>>(J);
        svpf::add_launches(1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && n > 0) {
        dim3 grid((unsigned)((n + 255) / 256 < 65535 ? (n + 255) / 256 : 65535), (unsigned)npayloads);
        mask_finish_kernel<<<grid, 256, 0, st>>>(J);
        svpf::add_launches(1);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        svpf::set_last_error(std::string("mask planes: ") + cudaGetErrorString(e));
        return SVPF_ECUDA;
    }
    return SVPF_OK;
}

}  // extern "C"

extern "C" {

int svpf_scene_class_device(const int32_t *vdata, const uint8_t *payloads_dev, size_t payload_len, int32_t npayloads,
                            double luma_gamma, const svpf_scene_limits *limits, int32_t *classes_dev,
                            int32_t *status_dev, void *stream) {
    if (int rc = svpf::require_device()) return rc;
    VecHdr h;
    if (!read_vdata(vdata, h) || !limits) {
        svpf::set_last_error(limits ? "not a vector header" : "null scene limits");
        return SVPF_EINVAL;
    }
    if (npayloads <= 0) return SVPF_OK;
    if (!payloads_dev || !classes_dev || !status_dev || payload_len < 0x40 || npayloads > (1 << 24)) {
        svpf::set_last_error("bad buffers");
        return SVPF_EINVAL;
    }
    if ((payload_len & 3) || ((uintptr_t)payloads_dev & 3)) {
        svpf::set_last_error("payloads must be 4-byte aligned");
        return SVPF_EINVAL;
    }
    SceneJob J;
    J.payloads = payloads_dev;
    J.payload_len = (int64_t)payload_len;
    J.classes = classes_dev;
    J.status = status_dev;
    J.flags = h.flags;
    J.gw = h.gw > 0 ? h.gw : 0;
    J.gh = h.gh > 0 ? h.gh : 0;
    J.blocks_pct = limits->blocks_pct;
    J.zero = limits->zero;
    J.m1 = limits->m1;
    J.m2 = limits->m2;
    J.scene = limits->scene;
    const double denom = h.marker == 3 ? 510.0 : 255.0;
    for (int k = 0; k < 512; k++) {  // luma_byte: (value^gamma * 255) as i32, .max(20) & 0xFF
        const double v = pow(((double)k) / denom, luma_gamma) * 255.0;
        const int32_t scaled = v != v ? 0 : (v >= 2147483647.0 ? INT32_MAX : (v <= -2147483648.0 ? INT32_MIN : (int32_t)v));
        J.luma[k] = (uint8_t)((scaled > 20 ? scaled : 20) & 0xFF);
    }
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(status_dev, 0, sizeof(int32_t) * (size_t)npayloads, st);
    if (e == cudaSuccess) {
        scene_class_kernel<<<(unsigned)npayloads * kSceneCtas, 256, 0, st>>>(J);
        svpf::add_launches(1);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        svpf::set_last_error(std::string("scene class: ") + cudaGetErrorString(e));
        return SVPF_ECUDA;
    }
    return SVPF_OK;
}

}  // extern "C"
