// capi.cpp -- the C ABI (include/svpflow_b200.h) over the Super / Analyse launchers.
//
// Host-buffer entry points own device buffers that grow on demand and are reused;
// device entry points take caller buffers and never allocate.
#include <cuda_runtime.h>
#include <string.h>

#include <mutex>
#include <string>
#include <vector>

#include "../../include/svpflow_b200.h"
#include "handles.h"
#include "svpf_device.h"

using namespace svpf;

namespace {

thread_local std::string g_err;
thread_local int64_t g_launches = 0;

int fail(int code, const std::string &msg) {
    g_err = msg;
    return code;
}
int cuda_fail(cudaError_t e, const char *where) {
    g_err = std::string(where) + ": " + cudaGetErrorString(e);
    return SVPF_ECUDA;
}
#define CU(call)                                               \
    do {                                                       \
        cudaError_t e_ = (call);                               \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call);    \
    } while (0)

int check_device() {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0)
        return fail(SVPF_ECUDA, "no CUDA device: the svpflow_b200 library computes on an NVIDIA GPU only");
    return SVPF_OK;
}

constexpr int64_t kStatusBytes = 256;
// level-0 look-ahead counters (4 x uint64) inside the status area, cleared with it
constexpr int64_t kStatsOffset = 64;
inline int64_t align256(int64_t v) { return (v + 255) & ~(int64_t)255; }

struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
    int ensure(size_t n) {
        if (n <= cap) return SVPF_OK;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        cudaError_t e = cudaMalloc(&p, n);
        if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc");
        cap = n;
        return SVPF_OK;
    }
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

}  // namespace

struct svpf_super {
    SuperOpts so;
    SuperLayout L;
    SuperDev D;
    std::mutex mu;
    DevBuf src, dst;
    cudaStream_t stream = nullptr;
    ~svpf_super() {
        if (stream) cudaStreamDestroy(stream);
    }
};

struct svpf_analyser {
    AnalyseOpts o;
    int32_t bits = 8;
    AnalyseParams P;
    SuperLayout L;
    int32_t vdata[16];
    std::mutex mu;
    DevBuf supers, scratch, payloads, frames;
    cudaStream_t stream = nullptr;
    ~svpf_analyser() {
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

int make_super(const SuperOpts &so, svpf_super **out) {
    auto *s = new svpf_super;
    s->so = so;
    s->L = portable_layout(so);
    if (!make_super_dev(so, s->L, so.width, so.width / 2, s->D)) {
        delete s;
        return fail(SVPF_EINVAL, "unsupported super level count");
    }
    *out = s;
    return SVPF_OK;
}

int finish_analyser(svpf_analyser *a, svpf_analyser **out) {
    SuperOpts so;
    so.pel = a->o.pel;
    so.levels = a->o.super_levels;
    so.full = 1;
    so.width = a->o.width;
    so.height = a->o.height;
    so.bits = a->bits;
    a->L = portable_layout(so);
    std::string err;
    if (!build_analyse_params(a->o, a->L, a->P, err)) {
        delete a;
        return fail(err.find("not available") != std::string::npos ? SVPF_EUNSUP : SVPF_EINVAL, err);
    }
    vdata_header(a->o, a->vdata);
    *out = a;
    return SVPF_OK;
}

int ensure_stream(cudaStream_t &st) {
    if (!st) CU(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    return SVPF_OK;
}

// launches Analyse for `count` pairs given either explicitly (host table, staged into the
// scratch's head) or as a clip range computed on the device
int launch_pairs(const svpf_analyser *a, const PairRef *host_pairs, const uint8_t *clip, int32_t nframes, int32_t first,
                 int32_t count, uint8_t *payloads_dev, void *scratch_dev, cudaStream_t st) {
    uint8_t *scr = (uint8_t *)scratch_dev;
    const int64_t table = align256((int64_t)count * (int64_t)sizeof(PairRef));
    CU(cudaMemsetAsync(scr, 0, kStatusBytes, st));
    PairSrc src{};
    if (host_pairs) {
        PairRef *pairs_dev = (PairRef *)(scr + kStatusBytes);
        CU(cudaMemcpyAsync(pairs_dev, host_pairs, sizeof(PairRef) * (size_t)count, cudaMemcpyHostToDevice, st));
        src.table = pairs_dev;
    } else {
        src.clip = clip;
        src.frame_bytes = a->L.frame_bytes;
        src.first = first;
        src.nframes = nframes;
        src.delta = a->o.delta > 1 ? a->o.delta : 1;
    }
    src.stats = (unsigned long long *)(scr + kStatsOffset);
    int nl = 0;
    cudaError_t e = launch_analyse(a->P, src, count, payloads_dev, scr + kStatusBytes + table, (int *)scr, st, &nl);
    g_launches += nl;
    if (e != cudaSuccess) return cuda_fail(e, "analyse launch");
    return SVPF_OK;
}

int read_status(const void *scratch_dev, cudaStream_t st) {
    int status = 0;
    CU(cudaMemcpyAsync(&status, scratch_dev, sizeof(int), cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    if (status & 1) return fail(SVPF_EPANIC, "SVAnalyse: the reference indexes out of range on this input (it panics)");
    if (status & 4) return fail(SVPF_ECUDA, "SVAnalyse: an internal wait of the Analyse kernel gave up (results invalid)");
    if (status) return fail(SVPF_EUNSUP, "SVAnalyse: unsupported input on the device path");
    return SVPF_OK;
}

}  // namespace

namespace svpf {
// internals used by the other host translation units (handles.h)
const SuperOpts *super_opts_of(const svpf_super *s) { return &s->so; }
const SuperLayout *super_layout_of(const svpf_super *s) { return &s->L; }
const SuperDev *super_dev_of(const svpf_super *s) { return &s->D; }
const AnalyseOpts *analyser_opts(const svpf_analyser *a) { return &a->o; }
int require_device() { return check_device(); }
const AnalyseParams *analyser_params(const svpf_analyser *a) { return &a->P; }
const SuperLayout *analyser_layout(const svpf_analyser *a) { return &a->L; }
int32_t analyser_delta(const svpf_analyser *a) { return a->o.delta; }
void set_last_error(const std::string &msg) { g_err = msg; }
void add_launches(int n) { g_launches += n; }
}  // namespace svpf

extern "C" {

const char *svpf_last_error(void) { return g_err.c_str(); }
int64_t svpf_reference_version(void) { return 1174405393; }
int64_t svpf_kernel_launches(void) { return g_launches; }
void svpf_kernel_launches_reset(void) { g_launches = 0; }

int svpf_super_create(int32_t width, int32_t height, const char *opt, size_t opt_len, svpf_super **out) {
    if (!out) return fail(SVPF_EINVAL, "null output handle");
    if (width <= 0 || height <= 0) return fail(SVPF_EINVAL, "SVSuper: Clip must be YV12");
    OptTree tree;
    std::string err;
    const OptTree *t = nullptr;
    if (opt && opt_len > 0 && parse_opt(opt, opt_len, tree, err)) t = &tree;  // parse errors -> defaults
    SuperOpts so;
    if (!super_opts_from_opt(t, width, height, so, err)) return fail(SVPF_EINVAL, err);
    return make_super(so, out);
}

int svpf_super_create_bits(int32_t width, int32_t height, const char *opt, size_t opt_len, int32_t bits,
                           svpf_super **out) {
    if (!out) return fail(SVPF_EINVAL, "null output handle");
    if (bits != 8 && bits != 10) return fail(SVPF_EINVAL, "bits must be 8 or 10");
    if (width <= 0 || height <= 0) return fail(SVPF_EINVAL, "SVSuper: Clip must be YV12");
    OptTree tree;
    std::string err;
    const OptTree *t = nullptr;
    if (opt && opt_len > 0 && parse_opt(opt, opt_len, tree, err)) t = &tree;
    SuperOpts so;
    if (!super_opts_from_opt(t, width, height, so, err)) return fail(SVPF_EINVAL, err);
    so.bits = bits;
    return make_super(so, out);
}

int svpf_super_create_portable(int32_t width, int32_t height, int32_t pel, svpf_super **out) {
    if (!out) return fail(SVPF_EINVAL, "null output handle");
    if (!(pel == 1 || pel == 2 || pel == 4)) return fail(SVPF_EINVAL, "pel must be 1, 2 or 4");
    if (width <= 0 || height <= 0 || width % 2 != 0 || height % 2 != 0)
        return fail(SVPF_EINVAL, "dimensions must be positive and even");
    SuperOpts so;
    std::string err;
    if (!super_opts_from_opt(nullptr, width, height, so, err)) return fail(SVPF_EINVAL, err);
    so.pel = pel;
    return make_super(so, out);
}

void svpf_super_destroy(svpf_super *s) { delete s; }
int64_t svpf_super_sdata(const svpf_super *s) { return super_pack_data(s->so); }
int32_t svpf_super_height(const svpf_super *s) { return s->L.super_h; }
int32_t svpf_super_levels(const svpf_super *s) { return s->so.levels; }
int32_t svpf_super_pel(const svpf_super *s) { return s->so.pel; }
size_t svpf_super_source_len(const svpf_super *s) {
    size_t w = (size_t)s->so.width, h = (size_t)s->so.height;
    return (w * h + 2 * ((w / 2) * (h / 2))) * (size_t)s->L.px_bytes;
}
int32_t svpf_super_bits(const svpf_super *s) { return s->so.bits; }
size_t svpf_super_output_len(const svpf_super *s) { return (size_t)s->L.frame_bytes; }

int svpf_super_build_device(const svpf_super *s, const uint8_t *src_dev, int64_t src_y_stride, int64_t src_c_stride,
                            uint8_t *dst_dev, int32_t nframes, void *stream) {
    if (int rc = check_device()) return rc;
    if (nframes < 0 || (nframes > 0 && (!src_dev || !dst_dev))) return fail(SVPF_EINVAL, "bad buffers");
    if (s->L.px_bytes == 2 && (((uintptr_t)src_dev | (uintptr_t)dst_dev) & 1))
        return fail(SVPF_EINVAL, "16-bit frames must be 2-byte aligned");
    SuperDev D = s->D;
    if (src_y_stride > 0 || src_c_stride > 0) {
        if (src_y_stride < s->so.width || src_c_stride < s->so.width / 2) return fail(SVPF_EINVAL, "source pitch below width");
        if (!make_super_dev(s->so, s->L, src_y_stride, src_c_stride, D)) return fail(SVPF_EINVAL, "bad layout");
    }
    int nl = 0;
    cudaError_t e = launch_super(D, src_dev, dst_dev, nframes, (cudaStream_t)stream, &nl);
    g_launches += nl;
    if (e != cudaSuccess) return cuda_fail(e, "super launch");
    return SVPF_OK;
}

int svpf_super_build(const svpf_super *cs, const uint8_t *src, uint8_t *dst, int32_t nframes) {
    if (int rc = check_device()) return rc;
    if (nframes <= 0) return SVPF_OK;
    svpf_super *s = const_cast<svpf_super *>(cs);
    std::lock_guard<std::mutex> lk(s->mu);
    if (int rc = ensure_stream(s->stream)) return rc;
    const size_t in = svpf_super_source_len(s) * (size_t)nframes, outb = (size_t)s->L.frame_bytes * (size_t)nframes;
    if (int rc = s->src.ensure(in)) return rc;
    if (int rc = s->dst.ensure(outb)) return rc;
    CU(cudaMemcpyAsync(s->src.p, src, in, cudaMemcpyHostToDevice, s->stream));
    int nl = 0;
    cudaError_t e = launch_super(s->D, (const uint8_t *)s->src.p, (uint8_t *)s->dst.p, nframes, s->stream, &nl);
    g_launches += nl;
    if (e != cudaSuccess) return cuda_fail(e, "super launch");
    CU(cudaMemcpyAsync(dst, s->dst.p, outb, cudaMemcpyDeviceToHost, s->stream));
    CU(cudaStreamSynchronize(s->stream));
    return SVPF_OK;
}

int svpf_analyser_create(int64_t sdata, const char *opt, size_t opt_len, int32_t src_width, int32_t src_height,
                         svpf_analyser **out) {
    if (!out) return fail(SVPF_EINVAL, "null output handle");
    OptTree tree;
    std::string err;
    const OptTree *t = nullptr;
    if (opt && opt_len > 0 && parse_opt(opt, opt_len, tree, err)) t = &tree;
    auto *a = new svpf_analyser;
    if (!analyse_opts_from_opt(t, sdata, nullptr, a->o, err)) {
        delete a;
        return fail(SVPF_EINVAL, err);
    }
    if (src_width > 0) a->o.width = src_width;
    if (src_height > 0) a->o.height = src_height;
    return finish_analyser(a, out);
}

int svpf_analyser_create_portable(const svpf_super *s, int32_t bw, int32_t bh, int32_t overlap_mode, int32_t vectors,
                                  svpf_analyser **out) {
    if (!out || !s) return fail(SVPF_EINVAL, "null handle");
    auto *a = new svpf_analyser;
    std::string err;
    if (!analyse_opts_portable(s->so, bw, bh, overlap_mode, vectors, a->o, err)) {
        delete a;
        return fail(SVPF_EINVAL, err);
    }
    return finish_analyser(a, out);
}

int svpf_analyser_create_bits(int64_t sdata, const char *opt, size_t opt_len, int32_t src_width, int32_t src_height,
                              int32_t bits, svpf_analyser **out) {
    if (!out) return fail(SVPF_EINVAL, "null output handle");
    if (bits != 8 && bits != 10) return fail(SVPF_EINVAL, "bits must be 8 or 10");
    OptTree tree;
    std::string err;
    const OptTree *t = nullptr;
    if (opt && opt_len > 0 && parse_opt(opt, opt_len, tree, err)) t = &tree;
    auto *a = new svpf_analyser;
    if (!analyse_opts_from_opt(t, sdata, nullptr, a->o, err)) {
        delete a;
        return fail(SVPF_EINVAL, err);
    }
    if (src_width > 0) a->o.width = src_width;
    if (src_height > 0) a->o.height = src_height;
    a->bits = bits;
    return finish_analyser(a, out);
}

void svpf_analyser_destroy(svpf_analyser *a) { delete a; }
const int32_t *svpf_analyser_vdata(const svpf_analyser *a) { return a->vdata; }
size_t svpf_analyser_payload_len(const svpf_analyser *a) { return (size_t)a->P.payload_len; }
int32_t svpf_analyser_delta(const svpf_analyser *a) { return a->o.delta; }
size_t svpf_analyser_scratch_bytes(const svpf_analyser *a, int32_t npairs) {
    if (npairs <= 0) return (size_t)kStatusBytes;
    return (size_t)(kStatusBytes + align256((int64_t)npairs * (int64_t)sizeof(PairRef)) + (int64_t)npairs * a->P.scratch_per_pair);
}

// The kernels write payload words (4 bytes), keep 8-byte fields in the scratch and read 16-bit
// samples as such: misaligned buffers would fault, so they are refused here.
static int check_alignment(const svpf_analyser *a, const uint8_t *super, const uint8_t *payloads, const void *scratch) {
    if (a->P.px_bytes == 2 && ((uintptr_t)super & 1)) return fail(SVPF_EINVAL, "16-bit super frames must be 2-byte aligned");
    if ((uintptr_t)payloads & 3) return fail(SVPF_EINVAL, "payloads must be 4-byte aligned");
    if ((uintptr_t)scratch & 15) return fail(SVPF_EINVAL, "scratch must be 16-byte aligned");
    return SVPF_OK;
}

int svpf_analyse_pairs_device(const svpf_analyser *a, const uint8_t *const *cur_dev, const uint8_t *const *ref_dev,
                              int32_t npairs, uint8_t *payloads_dev, void *scratch_dev, void *stream) {
    if (int rc = check_device()) return rc;
    if (npairs <= 0) return SVPF_OK;
    if (!cur_dev || !ref_dev || !payloads_dev || !scratch_dev) return fail(SVPF_EINVAL, "bad buffers");
    if (int rc = check_alignment(a, nullptr, payloads_dev, scratch_dev)) return rc;
    std::vector<PairRef> pr((size_t)npairs);
    for (int32_t i = 0; i < npairs; i++) {
        if (int rc = check_alignment(a, cur_dev[i], nullptr, nullptr)) return rc;
        if (int rc = check_alignment(a, ref_dev[i], nullptr, nullptr)) return rc;
        pr[(size_t)i] = PairRef{cur_dev[i], ref_dev[i]};
    }
    int rc = launch_pairs(a, pr.data(), nullptr, 0, 0, npairs, payloads_dev, scratch_dev, (cudaStream_t)stream);
    if (rc == SVPF_OK) CU(cudaStreamSynchronize((cudaStream_t)stream));  // the pair table is staged from `pr`
    return rc;
}

int svpf_clip_analyse_device(const svpf_analyser *a, const uint8_t *supers_dev, int32_t nframes, int32_t first,
                             int32_t count, uint8_t *payloads_dev, void *scratch_dev, void *stream) {
    if (int rc = check_device()) return rc;
    if (count <= 0) return SVPF_OK;
    if (first < 0 || first + count > nframes || !supers_dev || !payloads_dev || !scratch_dev)
        return fail(SVPF_EINVAL, "bad frame range or buffers");
    if (int rc = check_alignment(a, supers_dev, payloads_dev, scratch_dev)) return rc;
    return launch_pairs(a, nullptr, supers_dev, nframes, first, count, payloads_dev, scratch_dev, (cudaStream_t)stream);
}

int svpf_device_status(const void *scratch_dev, void *stream) {
    if (int rc = check_device()) return rc;
    return read_status(scratch_dev, (cudaStream_t)stream);
}

int svpf_analyser_set_lookahead(svpf_analyser *a, int32_t levels) {
    if (!a) return fail(SVPF_EINVAL, "null analyser");
    if (levels < 0 || levels > 7) return fail(SVPF_EINVAL, "look-ahead mode must be 0..7");
    std::lock_guard<std::mutex> lk(a->mu);
    a->P.lookahead = levels;
    return SVPF_OK;
}

int svpf_device_lookahead_stats(const void *scratch_dev, void *stream, int64_t out[4]) {
    if (int rc = check_device()) return rc;
    if (!scratch_dev || !out) return fail(SVPF_EINVAL, "bad buffers");
    unsigned long long v[4] = {0, 0, 0, 0};
    CU(cudaMemcpyAsync(v, (const uint8_t *)scratch_dev + kStatsOffset, sizeof(v), cudaMemcpyDeviceToHost,
                       (cudaStream_t)stream));
    CU(cudaStreamSynchronize((cudaStream_t)stream));
    for (int i = 0; i < 4; i++) out[i] = (int64_t)v[i];
    return SVPF_OK;
}

int svpf_analyse(svpf_analyser *a, const uint8_t *cur_super, const uint8_t *ref_super, uint8_t *payload) {
    if (int rc = check_device()) return rc;
    std::lock_guard<std::mutex> lk(a->mu);
    if (int rc = ensure_stream(a->stream)) return rc;
    const size_t fb = (size_t)a->L.frame_bytes;
    if (int rc = a->supers.ensure(2 * fb)) return rc;
    if (int rc = a->scratch.ensure(svpf_analyser_scratch_bytes(a, 1))) return rc;
    if (int rc = a->payloads.ensure((size_t)a->P.payload_len)) return rc;
    uint8_t *d = (uint8_t *)a->supers.p;
    CU(cudaMemcpyAsync(d, cur_super, fb, cudaMemcpyHostToDevice, a->stream));
    CU(cudaMemcpyAsync(d + fb, ref_super, fb, cudaMemcpyHostToDevice, a->stream));
    PairRef pr{d, d + fb};
    if (int rc = launch_pairs(a, &pr, nullptr, 0, 0, 1, (uint8_t *)a->payloads.p, a->scratch.p, a->stream)) return rc;
    CU(cudaMemcpyAsync(payload, a->payloads.p, (size_t)a->P.payload_len, cudaMemcpyDeviceToHost, a->stream));
    return read_status(a->scratch.p, a->stream);
}

int svpf_clip_analyse(svpf_analyser *a, const svpf_super *s, const uint8_t *frames, int32_t nframes, int32_t first,
                      int32_t count, uint8_t *payloads) {
    if (int rc = check_device()) return rc;
    if (count <= 0) return SVPF_OK;
    if (first < 0 || first + count > nframes) return fail(SVPF_EINVAL, "bad frame range");
    if (s->L.frame_bytes != a->L.frame_bytes) return fail(SVPF_EINVAL, "super frame configuration mismatch");
    std::lock_guard<std::mutex> lk(a->mu);
    if (int rc = ensure_stream(a->stream)) return rc;
    const size_t src_fb = svpf_super_source_len(s), fb = (size_t)a->L.frame_bytes;
    if (int rc = a->frames.ensure(src_fb * (size_t)nframes)) return rc;
    if (int rc = a->supers.ensure(fb * (size_t)nframes)) return rc;
    if (int rc = a->scratch.ensure(svpf_analyser_scratch_bytes(a, count))) return rc;
    if (int rc = a->payloads.ensure((size_t)a->P.payload_len * (size_t)count)) return rc;
    CU(cudaMemcpyAsync(a->frames.p, frames, src_fb * (size_t)nframes, cudaMemcpyHostToDevice, a->stream));
    int nl = 0;
    cudaError_t e = launch_super(s->D, (const uint8_t *)a->frames.p, (uint8_t *)a->supers.p, nframes, a->stream, &nl);
    g_launches += nl;
    if (e != cudaSuccess) return cuda_fail(e, "super launch");
    if (int rc = launch_pairs(a, nullptr, (const uint8_t *)a->supers.p, nframes, first, count, (uint8_t *)a->payloads.p,
                              a->scratch.p, a->stream))
        return rc;
    CU(cudaMemcpyAsync(payloads, a->payloads.p, (size_t)a->P.payload_len * (size_t)count, cudaMemcpyDeviceToHost,
                       a->stream));
    return read_status(a->scratch.p, a->stream);
}

}  // extern "C"
