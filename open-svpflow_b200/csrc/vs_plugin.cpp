// vs_plugin.cpp -- the VapourSynth plugin (libsvpflow1_vs.so): the reference plugin's two
// exports and two filters, with Super and Analyse computed on the GPU.
//
// Follows crates/svpflow1/src/abi.rs (exports, plugin identity and registration strings),
// vs.rs (the VSAPI function-pointer offsets read here, the VideoInfo layout, activation
// reasons, FM_PARALLEL), super_filter.rs (Super: arguments, error texts, the `data` int,
// output video info, zeroed output planes built at the output frame's row pitches) and
// analyse_filter.rs (Analyse: arguments, error texts, the `data` int holding the address
// of the 16-int vector header, the Gray8 payload frames, frame n paired with
// min(n + delta, num_frames - 1)).
//
// The frame server calls getFrame from many threads (FM_PARALLEL). Each calling thread has
// its own CUDA stream and device buffers; a filter's state is read-only after creation.
// Super frames keep the frame server's row pitches on the device too, because the
// reference's results depend on them (the level-0 rows are edge-extended into the row
// padding, which the half-pel planes then read).
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <mutex>
#include <string>

#include "../../include/svpflow_b200.h"
#include "handles.h"
#include "svpf_device.h"

using namespace svpf;

namespace {

typedef void *Raw;
typedef const void *ConstRaw;

struct VideoInfo {  // vs.rs:76-86
    ConstRaw format;
    int64_t fps_num, fps_den;
    int32_t width, height, num_frames, flags;
};

typedef intptr_t (*CreateFn)(ConstRaw, Raw, Raw, Raw, ConstRaw);
typedef void (*ConfigFn)(const char *, const char *, const char *, int32_t, int32_t, Raw);
typedef void (*RegisterFn)(const char *, const char *, CreateFn, Raw, Raw);
typedef void (*InitFn)(ConstRaw, Raw, Raw *, Raw, Raw, ConstRaw);
typedef ConstRaw (*GetFrameCb)(int32_t, int32_t, Raw *, Raw *, Raw, Raw, ConstRaw);
typedef void (*FreeCb)(Raw, Raw, ConstRaw);
typedef void (*CreateFilterFn)(ConstRaw, Raw, const char *, InitFn, GetFrameCb, FreeCb, int32_t, int32_t, Raw, Raw);
typedef void (*SetErrorFn)(Raw, const char *);
typedef const VideoInfo *(*GetVideoInfoFn)(Raw);
typedef void (*SetVideoInfoFn)(const VideoInfo *, int32_t, Raw);
typedef int64_t (*PropGetIntFn)(ConstRaw, const char *, int32_t, int32_t *);
typedef const char *(*PropGetDataFn)(ConstRaw, const char *, int32_t, int32_t *);
typedef int32_t (*PropGetDataSizeFn)(ConstRaw, const char *, int32_t, int32_t *);
typedef Raw (*PropGetNodeFn)(ConstRaw, const char *, int32_t, int32_t *);
typedef int32_t (*PropSetIntFn)(Raw, const char *, int64_t, int32_t);
typedef void (*FreeFrameFn)(ConstRaw);
typedef void (*FreeNodeFn)(Raw);
typedef ConstRaw (*GetFrameFilterFn)(int32_t, Raw, Raw);
typedef Raw (*NewVideoFrameFn)(ConstRaw, int32_t, int32_t, ConstRaw, Raw);
typedef int32_t (*GetStrideFn)(ConstRaw, int32_t);
typedef const uint8_t *(*GetReadPtrFn)(ConstRaw, int32_t);
typedef uint8_t *(*GetWritePtrFn)(Raw, int32_t);
typedef void (*RequestFrameFilterFn)(int32_t, Raw, Raw);
typedef ConstRaw (*GetFormatPresetFn)(int32_t, Raw);

// byte offsets of the VSAPI entries (vs.rs:48-65, analyse_filter.rs:194)
constexpr size_t FREE_FRAME = 48, FREE_NODE = 56, NEW_VIDEO_FRAME = 72, CREATE_FILTER = 136, SET_ERROR = 144,
                 GET_FORMAT_PRESET = 176, GET_FRAME_FILTER = 208, REQUEST_FRAME_FILTER = 216, GET_STRIDE = 240,
                 GET_READ_PTR = 248, GET_WRITE_PTR = 256, GET_VIDEO_INFO = 304, SET_VIDEO_INFO = 312,
                 PROP_GET_INT = 392, PROP_GET_DATA = 408, PROP_GET_DATA_SIZE = 416, PROP_GET_NODE = 424,
                 PROP_SET_INT = 456;
constexpr int32_t AR_INITIAL = 0, AR_ALL_FRAMES_READY = 2, FM_PARALLEL = 100, PF_GRAY8 = 1000010;

template <class F>
F table_fn(ConstRaw vsapi, size_t off) {  // vs.rs:88-93 (unaligned read of a function pointer)
    F f = nullptr;
    if (vsapi) memcpy(&f, (const uint8_t *)vsapi + off, sizeof(f));
    return f;
}
void free_node(Raw node, ConstRaw vsapi) {
    if (!node) return;
    if (auto f = table_fn<FreeNodeFn>(vsapi, FREE_NODE)) f(node);
}
void set_error(Raw out, ConstRaw vsapi, const char *msg) {
    if (auto f = table_fn<SetErrorFn>(vsapi, SET_ERROR)) f(out, msg);
}
// The `opt` argument's bytes; an absent or empty value means none (super_filter.rs:107-121).
std::string read_opt(ConstRaw in, ConstRaw vsapi, bool *present) {
    *present = false;
    auto get_data = table_fn<PropGetDataFn>(vsapi, PROP_GET_DATA);
    auto get_size = table_fn<PropGetDataSizeFn>(vsapi, PROP_GET_DATA_SIZE);
    if (!get_data || !get_size) return {};
    int32_t err = 0;
    const char *p = get_data(in, "opt", 0, &err);
    if (!p || err) return {};
    const int32_t n = get_size(in, "opt", 0, &err);
    if (n <= 0) return {};
    *present = true;
    return std::string(p, (size_t)n);
}

// ---- per-thread device resources
struct DevCtx {
    int device = -1;
    cudaStream_t st = nullptr;
    uint8_t *buf = nullptr;
    size_t cap = 0;
    ~DevCtx() {
        if (st) cudaStreamSynchronize(st);
        if (buf) cudaFree(buf);
        if (st) cudaStreamDestroy(st);
    }
    uint8_t *get(size_t n) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (dev != device) {  // a context per thread and device
            if (st) cudaStreamDestroy(st);
            st = nullptr;
            buf = nullptr;
            cap = 0;
            device = dev;
        }
        if (!st && cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
        if (n > cap) {
            cudaStreamSynchronize(st);
            if (buf) cudaFree(buf);
            buf = nullptr;
            cap = 0;
            if (cudaMalloc(&buf, n) != cudaSuccess) return nullptr;
            cap = n;
        }
        return buf;
    }
};
thread_local DevCtx t_dev;

inline size_t al256(size_t v) { return (v + 255) & ~(size_t)255; }

// ======================================================================== Super
struct SuperFilter {
    Raw node;
    VideoInfo vi;
    SuperOpts so;
};

void init_super(ConstRaw, Raw, Raw *instance, Raw node, Raw, ConstRaw vsapi) {
    const SuperFilter *f = (const SuperFilter *)*instance;
    if (auto set_vi = table_fn<SetVideoInfoFn>(vsapi, SET_VIDEO_INFO)) set_vi(&f->vi, 1, node);
}

void free_super(Raw instance, Raw, ConstRaw vsapi) {
    SuperFilter *f = (SuperFilter *)instance;
    free_node(f->node, vsapi);
    delete f;
}

// The super frame of `src` written into `out` (both frame-server frames) on the GPU.
bool build_super_frame(const SuperFilter *f, ConstRaw src, Raw out, ConstRaw vsapi) {
    auto get_stride = table_fn<GetStrideFn>(vsapi, GET_STRIDE);
    auto get_read = table_fn<GetReadPtrFn>(vsapi, GET_READ_PTR);
    auto get_write = table_fn<GetWritePtrFn>(vsapi, GET_WRITE_PTR);
    const int64_t ys = get_stride(out, 0), cs = get_stride(out, 1);
    if (ys <= 0 || cs <= 0 || get_stride(out, 2) != cs) return false;  // one chroma pitch on the device
    const SuperOpts &so = f->so;
    const int64_t w = so.width, h = so.height, cw = w / 2, ch = h / 2;
    const SuperLayout L = strided_layout(so, ys, cs);
    SuperDev D;
    if (!make_super_dev(so, L, w, cw, D)) return false;
    const size_t src_bytes = (size_t)(w * h + 2 * cw * ch);
    uint8_t *dev = t_dev.get(al256(src_bytes) + (size_t)L.frame_bytes);
    if (!dev) return false;
    cudaStream_t st = t_dev.st;
    uint8_t *dsrc = dev, *dsup = dev + al256(src_bytes);
    cudaError_t e = cudaSuccess;
    for (int p = 0; p < 3 && e == cudaSuccess; p++) {  // packed source planes (their pitch does not matter)
        const uint8_t *sp = get_read(src, p);
        const int64_t sst = get_stride(src, p);
        const int64_t pw = p ? cw : w, ph = p ? ch : h;
        if (!sp || sst < pw) return false;
        uint8_t *d = dsrc + (p == 0 ? 0 : w * h + (p - 1) * cw * ch);
        if (pw > 0 && ph > 0) e = cudaMemcpy2DAsync(d, (size_t)pw, sp, (size_t)sst, (size_t)pw, (size_t)ph, cudaMemcpyHostToDevice, st);
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(dsup, 0, (size_t)L.frame_bytes, st);  // the reference zeroes the frame first
    int nl = 0;
    if (e == cudaSuccess) e = launch_super(D, dsrc, dsup, 1, st, &nl);
    const int64_t rows[3] = {L.super_h, L.super_h / 2, L.super_h / 2};
    const int64_t off[3] = {0, L.y_len, L.y_len + L.c_len};
    for (int p = 0; p < 3 && e == cudaSuccess; p++) {
        uint8_t *dp = get_write(out, p);
        if (!dp) continue;
        e = cudaMemcpyAsync(dp, dsup + off[p], (size_t)((p ? cs : ys) * rows[p]), cudaMemcpyDeviceToHost, st);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e == cudaSuccess;
}

ConstRaw get_frame_super(int32_t n, int32_t activation, Raw *instance, Raw *, Raw frame_ctx, Raw core,
                         ConstRaw vsapi) {
    const SuperFilter *f = (const SuperFilter *)*instance;
    if (activation == AR_INITIAL) {
        if (auto req = table_fn<RequestFrameFilterFn>(vsapi, REQUEST_FRAME_FILTER)) req(n, f->node, frame_ctx);
        return nullptr;
    }
    if (activation != AR_ALL_FRAMES_READY) return nullptr;
    auto get_frame = table_fn<GetFrameFilterFn>(vsapi, GET_FRAME_FILTER);
    auto new_frame = table_fn<NewVideoFrameFn>(vsapi, NEW_VIDEO_FRAME);
    auto free_frame = table_fn<FreeFrameFn>(vsapi, FREE_FRAME);
    if (!get_frame || !new_frame || !table_fn<GetStrideFn>(vsapi, GET_STRIDE) ||
        !table_fn<GetReadPtrFn>(vsapi, GET_READ_PTR) || !table_fn<GetWritePtrFn>(vsapi, GET_WRITE_PTR))
        return nullptr;
    ConstRaw src = get_frame(n, f->node, frame_ctx);
    if (!src) return nullptr;
    Raw out = new_frame(f->vi.format, f->vi.width, f->vi.height, src, core);
    if (!out) {
        if (free_frame) free_frame(src);
        return nullptr;
    }
    const bool ok = build_super_frame(f, src, out, vsapi);
    if (free_frame) free_frame(src);
    if (!ok) {
        if (free_frame) free_frame(out);
        return nullptr;
    }
    return out;
}

intptr_t create_super(ConstRaw in, Raw out, Raw, Raw core, ConstRaw vsapi) {
    auto get_node = table_fn<PropGetNodeFn>(vsapi, PROP_GET_NODE);
    auto get_vi = table_fn<GetVideoInfoFn>(vsapi, GET_VIDEO_INFO);
    auto create_filter = table_fn<CreateFilterFn>(vsapi, CREATE_FILTER);
    auto prop_set_int = table_fn<PropSetIntFn>(vsapi, PROP_SET_INT);
    if (!get_node || !get_vi || !create_filter || !prop_set_int) {
        set_error(out, vsapi, "SVSuper: invalid VSAPI table");
        return 0;
    }
    int32_t err = 0;
    Raw node = get_node(in, "clip", 0, &err);
    if (!node) {
        set_error(out, vsapi, "SVSuper: clip is required");
        return 0;
    }
    const VideoInfo *vip = get_vi(node);
    if (!vip) {
        free_node(node, vsapi);
        set_error(out, vsapi, "SVSuper: invalid clip");
        return 0;
    }
    const VideoInfo vi = *vip;
    if (vi.width <= 0 || vi.height <= 0 || !vi.format) {
        free_node(node, vsapi);
        set_error(out, vsapi, "SVSuper: Clip must be YV12");
        return 0;
    }
    bool present = false;
    const std::string opt = read_opt(in, vsapi, &present);
    svpf_super *h = nullptr;
    if (svpf_super_create(vi.width, vi.height, present ? opt.data() : nullptr, present ? opt.size() : 0, &h) != SVPF_OK) {
        free_node(node, vsapi);
        set_error(out, vsapi, svpf_last_error());
        return 0;
    }
    prop_set_int(out, "data", svpf_super_sdata(h), 0);
    auto *f = new SuperFilter;
    f->node = node;
    f->vi = vi;
    f->vi.height = svpf_super_height(h);
    f->so = *super_opts_of(h);
    svpf_super_destroy(h);
    create_filter(in, out, "SVSuper", init_super, get_frame_super, free_super, FM_PARALLEL, 0, f, core);
    return 0;
}

// ======================================================================== Analyse
struct AnalyseFilter {
    Raw super_node, src_node;
    VideoInfo vi;
    int32_t super_rows;    // rows of the super clip's frames
    AnalyseOpts o;
    int32_t vdata[16];     // published through `data`; lives as long as the filter
    ConstRaw gray;
    int64_t payload_len;
};

void init_analyse(ConstRaw, Raw, Raw *instance, Raw node, Raw, ConstRaw vsapi) {
    const AnalyseFilter *f = (const AnalyseFilter *)*instance;
    if (auto set_vi = table_fn<SetVideoInfoFn>(vsapi, SET_VIDEO_INFO)) set_vi(&f->vi, 1, node);
}

void free_analyse(Raw instance, Raw, ConstRaw vsapi) {
    AnalyseFilter *f = (AnalyseFilter *)instance;
    free_node(f->super_node, vsapi);
    free_node(f->src_node, vsapi);
    delete f;
}

// The payload of the pair (f0, f1) of super frames on the GPU; false when it cannot be
// produced (the caller returns no frame, as the reference does on its failures).
bool analyse_frames(const AnalyseFilter *f, ConstRaw f0, ConstRaw f1, uint8_t *payload, ConstRaw vsapi) {
    auto get_stride = table_fn<GetStrideFn>(vsapi, GET_STRIDE);
    auto get_read = table_fn<GetReadPtrFn>(vsapi, GET_READ_PTR);
    const int64_t ys = get_stride(f0, 0), cs = get_stride(f0, 1);
    if (ys <= 0 || cs <= 0 || get_stride(f0, 2) != cs || get_stride(f1, 0) != ys || get_stride(f1, 1) != cs ||
        get_stride(f1, 2) != cs)
        return false;
    SuperOpts so;
    so.pel = f->o.pel;
    so.levels = f->o.super_levels;
    so.full = 1;  // load_super_planes reads the planes as a full pyramid (analyse_filter.rs:358-375)
    so.width = f->o.width;
    so.height = f->o.height;
    const SuperLayout L = strided_layout(so, ys, cs);
    AnalyseParams P;
    std::string err;
    if (!build_analyse_params(f->o, L, P, err)) return false;
    const size_t fb = al256((size_t)L.frame_bytes);
    const size_t scr = al256((size_t)P.scratch_per_pair);
    uint8_t *dev = t_dev.get(2 * fb + scr + al256((size_t)P.payload_len) + 256);
    if (!dev) return false;
    cudaStream_t st = t_dev.st;
    uint8_t *sup = dev, *dscr = dev + 2 * fb, *dpay = dscr + scr;
    int *status = (int *)(dpay + al256((size_t)P.payload_len));
    const int64_t rows[3] = {L.super_h, L.super_h / 2, L.super_h / 2};
    const int64_t have[3] = {f->super_rows, f->super_rows / 2, f->super_rows / 2};
    const int64_t off[3] = {0, L.y_len, L.y_len + L.c_len};
    cudaError_t e = cudaMemsetAsync(dev, 0, 2 * fb, st);
    for (int k = 0; k < 2 && e == cudaSuccess; k++) {
        ConstRaw fr = k ? f1 : f0;
        for (int p = 0; p < 3 && e == cudaSuccess; p++) {
            const uint8_t *sp = get_read(fr, p);
            if (!sp) return false;
            const int64_t r = rows[p] < have[p] ? rows[p] : have[p];
            if (r > 0) e = cudaMemcpyAsync(sup + k * fb + off[p], sp, (size_t)((p ? cs : ys) * r), cudaMemcpyHostToDevice, st);
        }
    }
    PairSrc src{};
    src.clip = sup;
    src.frame_bytes = (int64_t)fb;
    src.first = 0;
    src.nframes = 2;
    src.delta = 1;
    int nl = 0, hstatus = 0;
    if (e == cudaSuccess) e = cudaMemsetAsync(status, 0, sizeof(int), st);
    if (e == cudaSuccess) e = launch_analyse(P, src, 1, dpay, dscr, status, st, &nl);
    if (e == cudaSuccess) e = cudaMemcpyAsync(payload, dpay, (size_t)P.payload_len, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hstatus, status, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e == cudaSuccess && hstatus == 0;
}

ConstRaw get_frame_analyse(int32_t n, int32_t activation, Raw *instance, Raw *, Raw frame_ctx, Raw core,
                           ConstRaw vsapi) {
    const AnalyseFilter *f = (const AnalyseFilter *)*instance;
    const int32_t delta = f->o.delta > 1 ? f->o.delta : 1;
    if (activation == AR_INITIAL) {
        if (auto req = table_fn<RequestFrameFilterFn>(vsapi, REQUEST_FRAME_FILTER)) {
            req(n, f->super_node, frame_ctx);
            req(n + delta, f->super_node, frame_ctx);
        }
        return nullptr;
    }
    if (activation != AR_ALL_FRAMES_READY) return nullptr;
    auto get_frame = table_fn<GetFrameFilterFn>(vsapi, GET_FRAME_FILTER);
    auto new_frame = table_fn<NewVideoFrameFn>(vsapi, NEW_VIDEO_FRAME);
    auto get_stride = table_fn<GetStrideFn>(vsapi, GET_STRIDE);
    auto get_write = table_fn<GetWritePtrFn>(vsapi, GET_WRITE_PTR);
    auto free_frame = table_fn<FreeFrameFn>(vsapi, FREE_FRAME);
    if (!get_frame || !new_frame || !get_stride || !table_fn<GetReadPtrFn>(vsapi, GET_READ_PTR) || !get_write)
        return nullptr;
    const int32_t last = f->vi.num_frames == INT32_MIN ? INT32_MIN : f->vi.num_frames - 1;  // saturating_sub(1)
    const int32_t n2 = (int64_t)n + delta < last ? n + delta : last;
    ConstRaw f0 = get_frame(n, f->super_node, frame_ctx);
    ConstRaw f1 = get_frame(n2, f->super_node, frame_ctx);
    auto release = [&] {
        if (!free_frame) return;
        if (f0) free_frame(f0);
        if (f1) free_frame(f1);
    };
    if (!f0 || !f1) {
        release();
        return nullptr;
    }
    std::string payload((size_t)f->payload_len, '\0');
    if (!analyse_frames(f, f0, f1, (uint8_t *)&payload[0], vsapi)) {
        release();
        return nullptr;
    }
    Raw out = new_frame(f->gray, (int32_t)f->payload_len, 1, f0, core);
    if (!out) {
        release();
        return nullptr;
    }
    const int32_t stride = get_stride(out, 0);
    uint8_t *p = get_write(out, 0);
    if (p && stride > 0) {
        const size_t ncopy = payload.size() < (size_t)stride ? payload.size() : (size_t)stride;
        memcpy(p, payload.data(), ncopy);
        if ((size_t)stride > ncopy) memset(p + ncopy, 0, (size_t)stride - ncopy);
    }
    release();
    return out;
}

intptr_t create_analyse(ConstRaw in, Raw out, Raw, Raw core, ConstRaw vsapi) {
    auto get_node = table_fn<PropGetNodeFn>(vsapi, PROP_GET_NODE);
    auto get_vi = table_fn<GetVideoInfoFn>(vsapi, GET_VIDEO_INFO);
    auto create_filter = table_fn<CreateFilterFn>(vsapi, CREATE_FILTER);
    auto prop_set_int = table_fn<PropSetIntFn>(vsapi, PROP_SET_INT);
    auto get_int = table_fn<PropGetIntFn>(vsapi, PROP_GET_INT);
    if (!get_node || !get_vi || !create_filter || !prop_set_int || !get_int) {
        set_error(out, vsapi, "SVAnalyse: invalid VSAPI");
        return 0;
    }
    int32_t err = 0;
    Raw super_node = get_node(in, "clip", 0, &err);
    if (!super_node) {
        set_error(out, vsapi, "SVAnalyse: clip (super) required");
        return 0;
    }
    Raw src_node = get_node(in, "src", 0, &err);
    if (!src_node) {
        free_node(super_node, vsapi);
        set_error(out, vsapi, "SVAnalyse: src required");
        return 0;
    }
    err = 0;
    const int64_t sdata = get_int(in, "sdata", 0, &err);
    if (err != 0) {
        free_node(super_node, vsapi);
        free_node(src_node, vsapi);
        set_error(out, vsapi, "SVAnalyse: sdata required");
        return 0;
    }
    const VideoInfo *src_vip = get_vi(src_node), *super_vip = get_vi(super_node);
    if (!src_vip || !super_vip) {
        free_node(super_node, vsapi);
        free_node(src_node, vsapi);
        set_error(out, vsapi, "SVAnalyse: invalid VSAPI");
        return 0;
    }
    const VideoInfo src_vi = *src_vip, super_vi = *super_vip;
    bool present = false;
    const std::string opt = read_opt(in, vsapi, &present);
    svpf_analyser *h = nullptr;
    const int rc = svpf_analyser_create(sdata, present ? opt.data() : nullptr, present ? opt.size() : 0,
                                        src_vi.width > 0 ? src_vi.width : 0, src_vi.height > 0 ? src_vi.height : 0, &h);
    if (rc != SVPF_OK) {
        free_node(super_node, vsapi);
        free_node(src_node, vsapi);
        set_error(out, vsapi, svpf_last_error());
        return 0;
    }
    ConstRaw gray = nullptr;
    if (auto gp = table_fn<GetFormatPresetFn>(vsapi, GET_FORMAT_PRESET)) gray = gp(PF_GRAY8, core);
    if (!gray) gray = super_vi.format;
    if (!gray) {
        svpf_analyser_destroy(h);
        free_node(super_node, vsapi);
        free_node(src_node, vsapi);
        set_error(out, vsapi, "SVAnalyse: cannot get Gray8 format");
        return 0;
    }
    auto *f = new AnalyseFilter;
    f->super_node = super_node;
    f->src_node = src_node;
    f->super_rows = super_vi.height;
    f->o = *analyser_opts(h);
    memcpy(f->vdata, svpf_analyser_vdata(h), sizeof(f->vdata));
    f->gray = gray;
    f->payload_len = (int64_t)svpf_analyser_payload_len(h);
    svpf_analyser_destroy(h);
    prop_set_int(out, "data", (int64_t)(intptr_t)f->vdata, 0);
    f->vi.format = gray;
    f->vi.fps_num = src_vi.fps_num;
    f->vi.fps_den = src_vi.fps_den;
    f->vi.width = (int32_t)f->payload_len;
    f->vi.height = 1;
    f->vi.num_frames = src_vi.num_frames;
    f->vi.flags = 0;
    if (super_vi.num_frames > 0 && super_vi.num_frames < f->vi.num_frames) f->vi.num_frames = super_vi.num_frames;
    create_filter(in, out, "SVAnalyse", init_analyse, get_frame_analyse, free_analyse, FM_PARALLEL, 0, f, core);
    return 0;
}

}  // namespace

extern "C" {

// svpGetVersion, crates/svpflow1/src/abi.rs:5-8
__attribute__((visibility("default"))) int64_t svpGetVersion(void) { return 1174405393; }

// VapourSynthPluginInit, crates/svpflow1/src/abi.rs:10-47
__attribute__((visibility("default"))) void VapourSynthPluginInit(ConfigFn config, RegisterFn reg, Raw plugin) {
    if (!config) return;
    config("com.svp-team.flow1", "svp1", "SVPFlow1", 0x30002, 1, plugin);
    if (!reg) return;
    reg("Super", "clip:clip;opt:data", create_super, nullptr, plugin);
    reg("Analyse", "clip:clip;sdata:int;src:clip;opt:data", create_analyse, nullptr, plugin);
}

}  // extern "C"
