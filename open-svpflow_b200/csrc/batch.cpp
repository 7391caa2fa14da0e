// batch.cpp -- the batched form: many clips of uneven size and length analysed by one
// persistent launch.
//
// The reference analyses one clip at a time, one output frame per getFrame call
// (crates/svpflow1/src/analyse_filter.rs:229-334); every frame pair is independent of
// every other (analyse_search.rs:68-92 reads only its two super frames). A batch therefore
// flattens the frame pairs of all its clips into one item list and lets a grid of
// resident CTAs drain it through a device-side counter (analyse_batch_kernel). The item
// list is sorted largest-first (longest-processing-time order) so that the small pairs
// fill the tail of the launch.
//
// Device memory of a batch is one allocation made at creation: every clip's source
// frames, super frames and payloads, the per-clip parameter blocks, the item list, a
// status word per clip and one search scratch slot per resident CTA. A run is one CUDA
// graph (the Super launches of every clip, the reset of the queue counter and the status
// words, the persistent Analyse launch) captured once per launch shape and replayed.
//
// The launch shape (threads per search direction, 4x4 tiles per lane) does not change
// any result; svpf_batch_autotune times the compiled shapes on the batch's largest items
// and keeps the fastest, remembered per device and clip mix (in-process, and in the
// file named by SVPF_TUNE_CACHE when set).
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/svpflow_b200.h"
#include "handles.h"
#include "svpf_device.h"

using namespace svpf;

namespace {

int bfail(int code, const std::string &msg) {
    set_last_error(msg);
    return code;
}
int bcuda(cudaError_t e, const char *where) { return bfail(SVPF_ECUDA, std::string(where) + ": " + cudaGetErrorString(e)); }
#define BCU(call)                                           \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) return bcuda(e_, #call);     \
    } while (0)

inline int64_t al256(int64_t v) { return (v + 255) & ~(int64_t)255; }

struct Tuned {
    int variant, tiles_per_lane;
};
std::mutex g_tune_mu;
std::map<std::string, Tuned> g_tune;
bool g_tune_loaded = false;

void tune_load_locked() {
    if (g_tune_loaded) return;
    g_tune_loaded = true;
    const char *path = getenv("SVPF_TUNE_CACHE");
    if (!path || !*path) return;
    FILE *f = fopen(path, "r");
    if (!f) return;
    char key[512];
    int v, t;
    while (fscanf(f, "%511s %d %d", key, &v, &t) == 3) g_tune[key] = Tuned{v, t};
    fclose(f);
}
void tune_store_locked() {
    const char *path = getenv("SVPF_TUNE_CACHE");
    if (!path || !*path) return;
    FILE *f = fopen(path, "w");
    if (!f) return;
    for (auto &kv : g_tune) fprintf(f, "%s %d %d\n", kv.first.c_str(), kv.second.variant, kv.second.tiles_per_lane);
    fclose(f);
}

}  // namespace

struct svpf_batch {
    struct Clip {
        SuperDev D;
        AnalyseParams P;
        int32_t nframes;
        int64_t src_frame_bytes, super_frame_bytes;
        int64_t frames_off, supers_off, payloads_off;
    };
    std::vector<Clip> clips;
    std::vector<BatchItem> items;  // device addresses, largest first
    std::vector<double> item_cost;
    uint8_t *arena = nullptr;
    int64_t arena_bytes = 0;
    int64_t off_params = 0, off_items = 0, off_counter = 0, off_status = 0, off_scratch = 0;
    int64_t scratch_per_cta = 0;
    int max_ctas = 0;          // scratch slots allocated
    int sms = 0;
    int variant = 3, tiles_per_lane = 8, grid = 0;  // nt128_b3 until tuned
    std::string signature;
    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_launches = 0;    // kernel launches inside one replay
    std::mutex mu;
    ~svpf_batch() {
        if (stream) cudaStreamSynchronize(stream);
        if (graph) cudaGraphExecDestroy(graph);
        if (stream) cudaStreamDestroy(stream);
        if (arena) cudaFree(arena);
    }
    AnalyseParams *params_dev() { return (AnalyseParams *)(arena + off_params); }
    BatchItem *items_dev() { return (BatchItem *)(arena + off_items); }
    unsigned *counter_dev() { return (unsigned *)(arena + off_counter); }
    int *status_dev() { return (int *)(arena + off_status); }
    uint8_t *scratch_dev() { return arena + off_scratch; }
};

namespace {

// The parameter blocks with the batch's tiles-per-lane knob, uploaded before a launch.
int upload_params(svpf_batch *b) {
    BCU(cudaStreamSynchronize(b->stream));  // no launch of this batch may still read the old blocks
    std::vector<AnalyseParams> ps(b->clips.size());
    for (size_t i = 0; i < b->clips.size(); i++) {
        ps[i] = b->clips[i].P;
        ps[i].tiles_per_lane = b->tiles_per_lane;
    }
    BCU(cudaMemcpy(b->params_dev(), ps.data(), sizeof(AnalyseParams) * ps.size(), cudaMemcpyHostToDevice));
    return SVPF_OK;
}

int grid_for(svpf_batch *b, int variant, int nitems, int *grid) {
    int per_sm = 0;
    BCU(analyse_variant(variant).batch_blocks_per_sm(&per_sm));
    if (per_sm <= 0) return bfail(SVPF_ECUDA, "batch kernel does not fit on an SM");
    int g = per_sm * b->sms;
    if (g > b->max_ctas) g = b->max_ctas;
    if (g > nitems) g = nitems;
    *grid = g;
    return SVPF_OK;
}

// Records the device work of one run on `st`: Super of every clip, queue and status reset,
// the persistent Analyse launch over the first `nitems` items.
int record_run(svpf_batch *b, cudaStream_t st, int nitems, int grid, int *launches) {
    int nl = 0;
    for (auto &c : b->clips) {
        cudaError_t e = launch_super(c.D, b->arena + c.frames_off, b->arena + c.supers_off, c.nframes, st, &nl);
        if (e != cudaSuccess) return bcuda(e, "super launch");
    }
    BCU(cudaMemsetAsync(b->counter_dev(), 0, 256, st));
    BCU(cudaMemsetAsync(b->status_dev(), 0, sizeof(int) * b->clips.size(), st));
    cudaError_t e = analyse_variant(b->variant).launch_batch(b->params_dev(), b->items_dev(), nitems, b->counter_dev(),
                                                             b->scratch_dev(), b->scratch_per_cta, b->status_dev(), grid,
                                                             st, &nl);
    if (e != cudaSuccess) return bcuda(e, "batch analyse launch");
    *launches = nl;
    return SVPF_OK;
}

int capture(svpf_batch *b) {
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    if (int rc = upload_params(b)) return rc;
    if (int rc = grid_for(b, b->variant, (int)b->items.size(), &b->grid)) return rc;
    cudaGraph_t g = nullptr;
    BCU(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    int nl = 0;
    int rc = record_run(b, b->stream, (int)b->items.size(), b->grid, &nl);
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return bcuda(e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return bcuda(e, "cudaGraphInstantiate");
    b->graph_launches = nl;
    return SVPF_OK;
}

int read_statuses(svpf_batch *b, cudaStream_t st) {
    std::vector<int> s(b->clips.size());
    BCU(cudaMemcpyAsync(s.data(), b->status_dev(), sizeof(int) * s.size(), cudaMemcpyDeviceToHost, st));
    BCU(cudaStreamSynchronize(st));
    for (size_t i = 0; i < s.size(); i++) {
        if (s[i] & 1)
            return bfail(SVPF_EPANIC, "SVAnalyse: clip " + std::to_string(i) +
                                          ": the reference indexes out of range on this input (it panics)");
        if (s[i]) return bfail(SVPF_EUNSUP, "SVAnalyse: clip " + std::to_string(i) + ": unsupported input on the device path");
    }
    return SVPF_OK;
}

}  // namespace

extern "C" {

int svpf_batch_create(int32_t nclips, const svpf_super *const *supers, const svpf_analyser *const *analysers,
                      const int32_t *nframes, svpf_batch **out) {
    if (!out) return bfail(SVPF_EINVAL, "null output handle");
    *out = nullptr;
    if (nclips <= 0 || !supers || !analysers || !nframes) return bfail(SVPF_EINVAL, "a batch needs at least one clip");
    if (int rc = require_device()) return rc;
    int dev = 0;
    cudaDeviceProp prop;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess)
        return bfail(SVPF_ECUDA, "cannot query the device");
    auto *b = new svpf_batch;
    b->sms = prop.multiProcessorCount;
    int64_t off = 0;
    int64_t max_scratch = 256;
    std::map<std::string, int> mix;
    char sig[96];
    for (int32_t i = 0; i < nclips; i++) {
        const svpf_super *s = supers[i];
        const svpf_analyser *a = analysers[i];
        if (!s || !a || nframes[i] <= 0) {
            delete b;
            return bfail(SVPF_EINVAL, "clip " + std::to_string(i) + ": null handle or no frames");
        }
        if (super_layout_of(s)->frame_bytes != analyser_layout(a)->frame_bytes) {
            delete b;
            return bfail(SVPF_EINVAL, "clip " + std::to_string(i) + ": super frame configuration mismatch");
        }
        if (super_layout_of(s)->px_bytes != 1 || analyser_layout(a)->px_bytes != 1) {
            delete b;
            return bfail(SVPF_EUNSUP, "clip " + std::to_string(i) + ": batches take 8-bit clips only");
        }
        svpf_batch::Clip c;
        c.D = *super_dev_of(s);
        c.P = *analyser_params(a);
        c.nframes = nframes[i];
        c.src_frame_bytes = c.D.src_frame_bytes;
        c.super_frame_bytes = c.D.frame_bytes;
        c.frames_off = off; off += al256(c.src_frame_bytes * c.nframes);
        c.supers_off = off; off += al256(c.super_frame_bytes * c.nframes);
        c.payloads_off = off; off += al256(c.P.payload_len * c.nframes);
        max_scratch = std::max(max_scratch, al256(c.P.scratch_per_pair));
        b->clips.push_back(c);
        snprintf(sig, sizeof(sig), "%dx%d/b%d/v%d/l%d", c.P.luma_w, c.P.luma_h, c.P.block_w, c.P.vectors, c.P.nlevels);
        mix[sig]++;
    }
    b->signature = std::string(prop.name) + "|";
    for (auto &kv : mix) b->signature += kv.first + ";";
    for (char &ch : b->signature)
        if (ch == ' ') ch = '_';
    // items: every output frame n of every clip pairs with min(n + delta, nframes - 1)
    for (int32_t i = 0; i < nclips; i++) {
        const auto &c = b->clips[(size_t)i];
        const int delta = std::max(c.P.header[15], 1);
        const double cost = (double)c.P.lv[0].gw * c.P.lv[0].gh * (c.P.lv[0].tl + 2.0 * c.P.lv[0].tc) *
                            (c.P.vectors == 3 ? 2.0 : 1.0);
        for (int32_t n = 0; n < c.nframes; n++) {
            const int32_t n2 = std::min(n + delta, c.nframes - 1);
            BatchItem it{};
            it.pair.cur = (const uint8_t *)(intptr_t)(c.supers_off + (int64_t)n * c.super_frame_bytes);
            it.pair.ref = (const uint8_t *)(intptr_t)(c.supers_off + (int64_t)n2 * c.super_frame_bytes);
            it.payload = (uint8_t *)(intptr_t)(c.payloads_off + (int64_t)n * c.P.payload_len);
            it.clip = i;
            b->items.push_back(it);
            b->item_cost.push_back(cost);
        }
    }
    {
        std::vector<size_t> order(b->items.size());
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) { return b->item_cost[x] > b->item_cost[y]; });
        std::vector<BatchItem> it2(order.size());
        std::vector<double> c2(order.size());
        for (size_t k = 0; k < order.size(); k++) { it2[k] = b->items[order[k]]; c2[k] = b->item_cost[order[k]]; }
        b->items.swap(it2);
        b->item_cost.swap(c2);
    }
    // the variant with the most resident CTAs bounds the scratch slots
    int most = 0;
    for (int v = 0; v < analyse_variant_count(); v++) {
        int per_sm = 0;
        if (analyse_variant(v).batch_blocks_per_sm(&per_sm) != cudaSuccess) {
            delete b;
            return bfail(SVPF_ECUDA, "occupancy query failed");
        }
        most = std::max(most, per_sm);
    }
    b->max_ctas = std::max(1, std::min<int>(most * b->sms, (int)b->items.size()));
    b->scratch_per_cta = max_scratch;
    b->off_params = off; off += al256((int64_t)sizeof(AnalyseParams) * nclips);
    b->off_items = off; off += al256((int64_t)sizeof(BatchItem) * (int64_t)b->items.size());
    b->off_counter = off; off += 256;
    b->off_status = off; off += al256((int64_t)sizeof(int) * nclips);
    b->off_scratch = off; off += max_scratch * b->max_ctas;
    b->arena_bytes = off;
    cudaError_t e = cudaMalloc(&b->arena, (size_t)off);
    if (e != cudaSuccess) {
        b->arena = nullptr;
        delete b;
        return bcuda(e, "cudaMalloc (batch arena)");
    }
    for (auto &it : b->items) {  // offsets -> device addresses
        it.pair.cur = b->arena + (intptr_t)it.pair.cur;
        it.pair.ref = b->arena + (intptr_t)it.pair.ref;
        it.payload = b->arena + (intptr_t)it.payload;
    }
    e = cudaMemcpy(b->items_dev(), b->items.data(), sizeof(BatchItem) * b->items.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete b;
        return bcuda(e, "batch set-up");
    }
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        tune_load_locked();
        auto f = g_tune.find(b->signature);
        if (f != g_tune.end() && f->second.variant >= 0 && f->second.variant < analyse_variant_count()) {
            b->variant = f->second.variant;
            b->tiles_per_lane = f->second.tiles_per_lane;
        }
    }
    if (int rc = capture(b)) {
        delete b;
        return rc;
    }
    *out = b;
    return SVPF_OK;
}

void svpf_batch_destroy(svpf_batch *b) { delete b; }
int32_t svpf_batch_clips(const svpf_batch *b) { return (int32_t)b->clips.size(); }
int64_t svpf_batch_pairs(const svpf_batch *b) { return (int64_t)b->items.size(); }
size_t svpf_batch_device_bytes(const svpf_batch *b) { return (size_t)b->arena_bytes; }
uint8_t *svpf_batch_frames_device(svpf_batch *b, int32_t clip) {
    if (clip < 0 || clip >= (int32_t)b->clips.size()) return nullptr;
    return b->arena + b->clips[(size_t)clip].frames_off;
}
const uint8_t *svpf_batch_payloads_device(const svpf_batch *b, int32_t clip) {
    if (clip < 0 || clip >= (int32_t)b->clips.size()) return nullptr;
    return b->arena + b->clips[(size_t)clip].payloads_off;
}
const char *svpf_batch_shape(const svpf_batch *b, int32_t *variant, int32_t *tiles_per_lane, int32_t *grid) {
    if (variant) *variant = b->variant;
    if (tiles_per_lane) *tiles_per_lane = b->tiles_per_lane;
    if (grid) *grid = b->grid;
    return analyse_variant(b->variant).name;
}
int32_t svpf_batch_graph_launches(const svpf_batch *b) { return b->graph_launches; }

int svpf_batch_set_shape(svpf_batch *b, int32_t variant, int32_t tiles_per_lane) {
    std::lock_guard<std::mutex> lk(b->mu);
    if (variant < 0 || variant >= analyse_variant_count()) return bfail(SVPF_EINVAL, "no such launch variant");
    if (!(tiles_per_lane == 2 || tiles_per_lane == 4 || tiles_per_lane == 8))
        return bfail(SVPF_EINVAL, "tiles per lane must be 2, 4 or 8");
    if (variant == b->variant && tiles_per_lane == b->tiles_per_lane && b->graph) return SVPF_OK;
    b->variant = variant;
    b->tiles_per_lane = tiles_per_lane;
    return capture(b);
}

int svpf_batch_launch(svpf_batch *b, void *stream) {
    std::lock_guard<std::mutex> lk(b->mu);
    cudaStream_t st = stream ? (cudaStream_t)stream : b->stream;
    BCU(cudaGraphLaunch(b->graph, st));
    add_launches(b->graph_launches);
    return SVPF_OK;
}

int svpf_batch_status(svpf_batch *b, void *stream) {
    std::lock_guard<std::mutex> lk(b->mu);
    return read_statuses(b, stream ? (cudaStream_t)stream : b->stream);
}

int svpf_batch_run(svpf_batch *b, const uint8_t *const *frames, uint8_t *const *payloads) {
    if (!frames || !payloads) return bfail(SVPF_EINVAL, "bad buffers");
    std::lock_guard<std::mutex> lk(b->mu);
    for (size_t i = 0; i < b->clips.size(); i++) {
        const auto &c = b->clips[i];
        if (!frames[i] || !payloads[i]) return bfail(SVPF_EINVAL, "clip " + std::to_string(i) + ": null buffer");
        BCU(cudaMemcpyAsync(b->arena + c.frames_off, frames[i], (size_t)(c.src_frame_bytes * c.nframes),
                            cudaMemcpyHostToDevice, b->stream));
    }
    BCU(cudaGraphLaunch(b->graph, b->stream));
    add_launches(b->graph_launches);
    for (size_t i = 0; i < b->clips.size(); i++) {
        const auto &c = b->clips[i];
        BCU(cudaMemcpyAsync(payloads[i], b->arena + c.payloads_off, (size_t)(c.P.payload_len * c.nframes),
                            cudaMemcpyDeviceToHost, b->stream));
    }
    return read_statuses(b, b->stream);
}

// Times each launch shape on the batch's largest items (one item per resident CTA of the
// shape, so a trial lasts about one pair's latency) and keeps the one with the most pairs
// per second. The source frames must be in place (svpf_batch_frames_device or a run).
int svpf_batch_autotune(svpf_batch *b, int32_t *variant, int32_t *tiles_per_lane, double *pairs_per_s) {
    std::lock_guard<std::mutex> lk(b->mu);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    BCU(cudaEventCreate(&e0));
    BCU(cudaEventCreate(&e1));
    auto trial = [&](int v, int t, double *rate) -> int {
        b->variant = v;
        b->tiles_per_lane = t;
        if (int rc = upload_params(b)) return rc;
        int grid = 0;
        if (int rc = grid_for(b, v, (int)b->items.size(), &grid)) return rc;
        const int n = grid;  // one item per resident CTA
        int nl = 0;
        for (auto &c : b->clips) {  // Super once (untimed), then the timed Analyse
            cudaError_t e = launch_super(c.D, b->arena + c.frames_off, b->arena + c.supers_off, c.nframes, b->stream, &nl);
            if (e != cudaSuccess) return bcuda(e, "super launch");
        }
        BCU(cudaMemsetAsync(b->counter_dev(), 0, 256, b->stream));
        BCU(cudaMemsetAsync(b->status_dev(), 0, sizeof(int) * b->clips.size(), b->stream));
        BCU(cudaEventRecord(e0, b->stream));
        cudaError_t e = analyse_variant(v).launch_batch(b->params_dev(), b->items_dev(), n, b->counter_dev(),
                                                        b->scratch_dev(), b->scratch_per_cta, b->status_dev(), grid,
                                                        b->stream, &nl);
        if (e != cudaSuccess) return bcuda(e, "batch analyse launch");
        BCU(cudaEventRecord(e1, b->stream));
        add_launches(nl);
        if (int rc = read_statuses(b, b->stream)) return rc;
        float ms = 0.f;
        BCU(cudaEventElapsedTime(&ms, e0, e1));
        *rate = ms > 0.f ? n * 1000.0 / ms : 0.0;
        return SVPF_OK;
    };
    int rc = SVPF_OK;
    double best = -1.0;
    int bv = 0, bt = 8;
    for (int v = 0; v < analyse_variant_count() && !rc; v++) {
        double r = 0;
        rc = trial(v, 8, &r);
        if (!rc && r > best) { best = r; bv = v; bt = 8; }
    }
    for (int t : {4, 2}) {
        if (rc) break;
        double r = 0;
        rc = trial(bv, t, &r);
        if (!rc && r > best) { best = r; bt = t; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    b->variant = bv;
    b->tiles_per_lane = bt;
    {
        std::lock_guard<std::mutex> lk2(g_tune_mu);
        g_tune[b->signature] = Tuned{bv, bt};
        tune_store_locked();
    }
    if (variant) *variant = bv;
    if (tiles_per_lane) *tiles_per_lane = bt;
    if (pairs_per_s) *pairs_per_s = best;
    return capture(b);
}

int32_t svpf_analyse_variant_count(void) { return analyse_variant_count(); }
const char *svpf_analyse_variant_name(int32_t i) {
    if (i < 0 || i >= analyse_variant_count()) return "";
    return analyse_variant(i).name;
}

}  // extern "C"
