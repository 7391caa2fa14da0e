// vectors.cu -- the consumer side of the Analyse payload on the device: decode the vectors
// and build the motion-vector planes a frame interpolator reads, without leaving HBM.
//
// Follows crates/svpflow-core/src/metadata.rs: vector_data (:89-115, the vdata header),
// motion_grid / extended_grid (:211-244), decode_vectors / decode_region (:246-273, :455-481);
// and renderer.rs: vector_planes (:1680-1726), clamp_to_frame (:1728-1736), sample_index
// (:1870-1874), centered (:3237-3243), as SmoothFps calls them (svpflow2 core.rs:962-1001): the
// "previous" set falls back to the current one and vice versa.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/svpflow_b200.h"
#include "handles.h"

namespace {

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

// grid: (positions / 256, payloads)
__global__ void vector_planes_kernel(const PlaneJob J) {
    const int64_t f = blockIdx.y;
    const uint8_t *p = J.payloads + f * J.payload_len;
    const int64_t count = (int64_t)J.gw * J.gh;
    const int64_t first = 0x40, second = first + 4 + count * 8;
    // decode_vectors' checks (every thread reads the same few words)
    bool ok = true;
    const bool hdr = rd32(p, J.payload_len, 0, ok) == 16 && rd32(p, J.payload_len, 4, ok) == 0xA0 &&
                     rd32(p, J.payload_len, 8, ok) == J.flags;
    const int marker = (int)(2 * count + 1);
    bool has_prev = (J.flags & 1) != 0, has_cur = (J.flags & 2) != 0;
    if (has_prev && rd32(p, J.payload_len, first, ok) != marker) ok = false;
    if (has_cur && rd32(p, J.payload_len, second, ok) != marker) ok = false;
    if (has_prev && first + 4 + count * 8 > J.payload_len) ok = false;
    if (has_cur && second + 4 + count * 8 > J.payload_len) ok = false;
    ok = ok && hdr && (has_prev || has_cur);
    if (!ok) {
        if (blockIdx.x == 0 && threadIdx.x == 0) J.status[f] = 1;
        return;
    }
    const int64_t off_prev = has_prev ? first + 4 : second + 4;  // previous falls back to current
    const int64_t off_cur = has_cur ? second + 4 : first + 4;    // and current to previous
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
    if (!payloads_dev || !planes_dev || !status_dev || payload_len < 0x40) {
        svpf::set_last_error("bad buffers");
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
