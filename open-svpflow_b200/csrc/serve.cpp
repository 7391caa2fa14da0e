// serve.cpp -- the served form: a request loop with continuous batching.
//
// Clips arrive at any time (svpf_server_submit). A scheduler thread admits them in
// arrival order while the device memory they need fits the server's HBM budget and an
// execution slot is free. An admitted clip gets a stream of its own and, in stream
// order: its source frames copied in, its super frames built (kept resident for all of
// its pairs: every super frame serves two adjacent pairs), its frame pairs analysed in
// chunks of `chunk_pairs`, each chunk's payloads copied out as soon as it finishes, and
// its memory released. A clip's chunks are spread over the slot's kLanes streams (they are
// independent frame pairs), and chunks of different clips run concurrently on the device, so a
// clip admitted while others are being analysed starts at once, and one that finishes
// frees its slot and memory for the next. Memory comes from the stream-ordered pool
// (cudaMallocAsync / cudaFreeAsync), so admission never synchronises the device.
//
// Per-pair completion times are taken by a host function queued behind each chunk's
// payload copy: the time the payload is in host memory. A clip's arrival time is taken at
// submit, so pair latency = done - arrival includes queueing for admission.
//
// Payloads go to page-locked memory directly. A pageable destination would make each
// copy wait for its chunk inside the scheduler thread, so those chunks land in the
// slot's page-locked staging buffer and the host function copies them out. No CUDA call
// is ever made while the server's lock is held: host functions take that lock, and a
// synchronising call (cudaFreeHost, cudaFree) under it could wait on them for ever.
//
// Results do not depend on the mix: every pair runs the same kernel on its own two super
// frames, whatever else shares the device.
#include <cuda_runtime.h>
#include <string.h>

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/svpflow_b200.h"
#include "handles.h"
#include "svpf_device.h"

using namespace svpf;

namespace {

inline int64_t al256(int64_t v) { return (v + 255) & ~(int64_t)255; }

constexpr int kCancelled = -2;  // Request::status of a request withdrawn before admission

constexpr int kLanes = 4;  // streams per slot: a clip's chunks run on them round-robin

struct Request;

struct Chunk {
    Request *req;
    int32_t first, count;
    uint8_t *stage;  // page-locked staging of the chunk's payloads, or null (copied to the destination directly)
};

struct Request {
    int64_t id = 0;
    SuperDev D;
    AnalyseParams P;
    int32_t nframes = 0, delta = 1;
    const uint8_t *frames = nullptr;
    uint8_t *payloads = nullptr;
    int64_t *pair_done_ns = nullptr;
    int64_t arrival_ns = 0, admit_ns = 0, done_ns = 0;
    int64_t need = 0;
    int slot = -1;
    uint8_t *dev = nullptr;
    bool pinned_out = false;     // payloads are page-locked host memory
    int status = 0;
    bool done = false;
    std::vector<Chunk> chunks;
    svpf_server *server = nullptr;
};

}  // namespace

struct svpf_server {
    int device = 0;
    int64_t budget = 0, used = 0, peak_used = 0;
    int max_active = 0, active = 0, peak_active = 0;
    int32_t chunk_pairs = 32;
    std::vector<cudaStream_t> streams;          // kLanes per slot
    std::vector<cudaEvent_t> events;            // kLanes + 1 per slot: lane joins, super frames ready
    std::vector<bool> slot_busy;
    int *slot_status = nullptr;                 // page-locked status word per slot
    std::vector<uint8_t *> stage;               // page-locked payload staging per slot (scheduler-owned)
    std::vector<size_t> stage_cap;
    std::vector<uint8_t *> retired;             // outgrown staging buffers, freed at destroy
    std::deque<Request *> pending;
    std::map<int64_t, std::unique_ptr<Request>> requests;
    int64_t next_id = 1, admitted = 0, completed = 0, cancelled = 0;
    std::atomic<int64_t> launches{0};
    std::mutex mu;
    std::condition_variable cv;       // scheduler wake-ups
    std::condition_variable done_cv;  // request completions
    bool stopping = false;
    std::thread worker;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    int64_t now_ns() const {
        return std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - t0).count();
    }
};

namespace {

int sfail(int code, const std::string &msg) {
    set_last_error(msg);
    return code;
}

int64_t lanes_of(const Request &r) { return r.chunks.size() < (size_t)kLanes ? (int64_t)r.chunks.size() : kLanes; }

int64_t request_bytes(const Request &r, int32_t chunk) {
    const int64_t c = chunk < r.nframes ? chunk : r.nframes;
    return al256(r.D.src_frame_bytes * r.nframes) + al256(r.D.frame_bytes * r.nframes) +
           al256(r.P.payload_len * r.nframes) + lanes_of(r) * al256(r.P.scratch_per_pair * c) + 256;
}

// Host function behind a chunk's payload copy (no CUDA calls allowed here).
void CUDART_CB chunk_done(void *arg) {
    Chunk *ch = (Chunk *)arg;
    Request *r = ch->req;
    svpf_server *s = r->server;
    if (ch->stage)
        memcpy(r->payloads + (int64_t)ch->first * r->P.payload_len, ch->stage, (size_t)(r->P.payload_len * ch->count));
    const int64_t t = s->now_ns();
    if (r->pair_done_ns)
        for (int32_t i = 0; i < ch->count; i++) r->pair_done_ns[ch->first + i] = t;
}

// Host function after the request's lanes have joined, its status word has been copied
// and its memory released.
void CUDART_CB request_done(void *arg) {
    Request *r = (Request *)arg;
    svpf_server *s = r->server;
    std::lock_guard<std::mutex> lk(s->mu);
    r->done_ns = s->now_ns();
    r->status = s->slot_status[r->slot];
    r->done = true;
    s->used -= r->need;
    s->active--;
    s->slot_busy[(size_t)r->slot] = false;
    s->completed++;
    s->cv.notify_all();
    s->done_cv.notify_all();
}

// Queues the whole of one admitted request on its slot's lanes: lane 0 allocates, copies the
// frames in and builds the super frames; every lane then analyses its chunks (own scratch,
// own staging) and copies their payloads out; lane 0 joins the lanes, copies the status word
// out, releases the memory and reports.
int enqueue(svpf_server *s, Request *r) {
    const int nl_lanes = (int)lanes_of(*r);
    cudaStream_t lane[kLanes];
    for (int k = 0; k < kLanes; k++) lane[k] = s->streams[(size_t)r->slot * kLanes + k];
    cudaStream_t st = lane[0];
    const int64_t fb = r->D.frame_bytes, sb = r->D.src_frame_bytes;
    const int64_t cmax = r->chunks.empty() ? 1 : r->chunks[0].count;
    cudaError_t e = cudaMallocAsync((void **)&r->dev, (size_t)r->need, st);
    if (e != cudaSuccess) {
        r->dev = nullptr;
        return SVPF_ECUDA;
    }
    uint8_t *frames = r->dev;
    uint8_t *supers = frames + al256(sb * r->nframes);
    uint8_t *pays = supers + al256(fb * r->nframes);
    uint8_t *scr0 = pays + al256(r->P.payload_len * r->nframes);
    const int64_t scr_lane = al256(r->P.scratch_per_pair * cmax);
    int *status = (int *)(scr0 + nl_lanes * scr_lane);
    uint8_t *stage[kLanes] = {nullptr, nullptr, nullptr, nullptr};
    if (!r->pinned_out) {  // this thread owns the slot's staging buffers while the slot is busy
        const size_t need = (size_t)(r->P.payload_len * cmax);
        for (int k = 0; k < nl_lanes; k++) {
            const size_t i = (size_t)r->slot * kLanes + k;
            if (s->stage_cap[i] < need) {
                if (s->stage[i]) s->retired.push_back(s->stage[i]);
                s->stage[i] = nullptr;
                s->stage_cap[i] = 0;
                if (cudaHostAlloc((void **)&s->stage[i], need, cudaHostAllocDefault) != cudaSuccess) return SVPF_ECUDA;
                s->stage_cap[i] = need;
            }
            stage[k] = s->stage[i];
        }
    }
    cudaEvent_t *ev = &s->events[(size_t)r->slot * (kLanes + 1)];
    int nl = 0;
    e = cudaMemsetAsync(status, 0, sizeof(int), st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(frames, r->frames, (size_t)(sb * r->nframes), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = launch_super(r->D, frames, supers, r->nframes, st, &nl);
    if (e == cudaSuccess) e = cudaEventRecord(ev[kLanes], st);
    for (int k = 1; k < nl_lanes && e == cudaSuccess; k++) e = cudaStreamWaitEvent(lane[k], ev[kLanes], 0);
    for (size_t k = 0; e == cudaSuccess && k < r->chunks.size(); k++) {
        Chunk &c = r->chunks[k];
        const int li = (int)(k % (size_t)nl_lanes);
        cudaStream_t ls = lane[li];
        PairSrc src{};
        src.clip = supers;
        src.frame_bytes = fb;
        src.first = c.first;
        src.nframes = r->nframes;
        src.delta = r->delta;
        e = launch_analyse_shape(kShapeShared, r->P, src, c.count, pays + (int64_t)c.first * r->P.payload_len,
                                 scr0 + li * scr_lane, status, ls, &nl);
        c.stage = stage[li];
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(c.stage ? c.stage : r->payloads + (int64_t)c.first * r->P.payload_len,
                                pays + (int64_t)c.first * r->P.payload_len, (size_t)(r->P.payload_len * c.count),
                                cudaMemcpyDeviceToHost, ls);
        if (e == cudaSuccess) e = cudaLaunchHostFunc(ls, chunk_done, &c);
    }
    for (int k = 1; k < nl_lanes && e == cudaSuccess; k++) {
        e = cudaEventRecord(ev[k], lane[k]);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(st, ev[k], 0);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&s->slot_status[r->slot], status, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaFreeAsync(r->dev, st);
    if (e == cudaSuccess) {
        r->dev = nullptr;
        e = cudaLaunchHostFunc(st, request_done, r);
    }
    s->launches += nl;
    return e == cudaSuccess ? SVPF_OK : SVPF_ECUDA;
}

void scheduler(svpf_server *s) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        s->cv.wait(lk, [&] {
            if (s->stopping) return true;
            if (s->pending.empty() || s->active >= s->max_active) return false;
            return s->used + s->pending.front()->need <= s->budget;
        });
        if (s->stopping) {  // requests never admitted fail
            for (Request *r : s->pending) {
                r->status = -1;
                r->done = true;
            }
            s->pending.clear();
            s->done_cv.notify_all();
            break;
        }
        Request *r = s->pending.front();
        s->pending.pop_front();
        int slot = 0;
        while (s->slot_busy[(size_t)slot]) slot++;
        s->slot_busy[(size_t)slot] = true;
        r->slot = slot;
        s->used += r->need;
        s->peak_used = s->used > s->peak_used ? s->used : s->peak_used;
        s->active++;
        s->peak_active = s->active > s->peak_active ? s->active : s->peak_active;
        s->admitted++;
        r->admit_ns = s->now_ns();
        lk.unlock();
        const int rc = enqueue(s, r);
        lk.lock();
        if (rc != SVPF_OK) {  // its last chunk will never report: wait out what was queued, release it here
            lk.unlock();
            for (int k = 0; k < kLanes; k++) cudaStreamSynchronize(s->streams[(size_t)slot * kLanes + k]);
            if (r->dev) cudaFree(r->dev);
            r->dev = nullptr;
            lk.lock();
            r->status = 4;
            r->done = true;
            r->done_ns = s->now_ns();
            s->used -= r->need;
            s->active--;
            s->slot_busy[(size_t)slot] = false;
            s->completed++;
            s->done_cv.notify_all();
        }
    }
}

}  // namespace

extern "C" {

int svpf_server_create(size_t hbm_budget_bytes, int32_t max_active, int32_t chunk_pairs, svpf_server **out) {
    if (!out) return sfail(SVPF_EINVAL, "null output handle");
    *out = nullptr;
    if (hbm_budget_bytes == 0 || max_active <= 0 || chunk_pairs <= 0)
        return sfail(SVPF_EINVAL, "budget, active clips and chunk size must be positive");
    if (int rc = require_device()) return rc;
    auto *s = new svpf_server;
    s->budget = (int64_t)hbm_budget_bytes;
    s->max_active = max_active;
    s->chunk_pairs = chunk_pairs;
    cudaGetDevice(&s->device);
    {  // keep freed blocks in the pool: clips come and go, their sizes repeat
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, s->device) == cudaSuccess) {
            uint64_t thr = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
        }
    }
    s->streams.assign((size_t)max_active * kLanes, nullptr);
    s->events.assign((size_t)max_active * (kLanes + 1), nullptr);
    s->slot_busy.assign((size_t)max_active, false);
    s->stage.assign((size_t)max_active * kLanes, nullptr);
    s->stage_cap.assign((size_t)max_active * kLanes, 0);
    cudaError_t e = cudaHostAlloc((void **)&s->slot_status, sizeof(int) * (size_t)max_active, cudaHostAllocDefault);
    for (auto &ev : s->events)
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    for (auto &st : s->streams)
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        for (auto &x : s->streams)
            if (x) cudaStreamDestroy(x);
        for (auto &x : s->events)
            if (x) cudaEventDestroy(x);
        if (s->slot_status) cudaFreeHost(s->slot_status);
        delete s;
        return sfail(SVPF_ECUDA, std::string("server set-up: ") + cudaGetErrorString(e));
    }
    s->worker = std::thread(scheduler, s);
    *out = s;
    return SVPF_OK;
}

int svpf_server_submit(svpf_server *s, const svpf_super *sup, const svpf_analyser *an, const uint8_t *frames,
                       int32_t nframes, uint8_t *payloads, int64_t *pair_done_ns, int64_t *request) {
    if (!s || !sup || !an || !frames || !payloads || nframes <= 0) return sfail(SVPF_EINVAL, "bad request");
    if (super_layout_of(sup)->frame_bytes != analyser_layout(an)->frame_bytes)
        return sfail(SVPF_EINVAL, "super frame configuration mismatch");
    if (super_layout_of(sup)->px_bytes != 1 || analyser_layout(an)->px_bytes != 1)
        return sfail(SVPF_EUNSUP, "the server takes 8-bit clips only");
    auto r = std::make_unique<Request>();
    r->arrival_ns = s->now_ns();
    r->D = *super_dev_of(sup);
    r->P = *analyser_params(an);
    r->nframes = nframes;
    r->delta = analyser_delta(an) > 1 ? analyser_delta(an) : 1;
    r->frames = frames;
    r->payloads = payloads;
    r->pair_done_ns = pair_done_ns;
    r->server = s;
    for (int32_t f = 0; f < nframes; f += s->chunk_pairs)
        r->chunks.push_back(Chunk{r.get(), f, (nframes - f) < s->chunk_pairs ? nframes - f : s->chunk_pairs});
    r->need = request_bytes(*r, s->chunk_pairs);
    if (r->need > s->budget) return sfail(SVPF_EINVAL, "clip needs more device memory than the server's budget");
    {
        cudaPointerAttributes pa;
        r->pinned_out = cudaPointerGetAttributes(&pa, payloads) == cudaSuccess && pa.type == cudaMemoryTypeHost;
        cudaGetLastError();  // a pageable pointer is not an error here
    }
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stopping) return sfail(SVPF_EINVAL, "server is shutting down");
    r->id = s->next_id++;
    if (request) *request = r->id;
    s->pending.push_back(r.get());
    s->requests[r->id] = std::move(r);
    s->cv.notify_all();
    return SVPF_OK;
}

int svpf_server_wait(svpf_server *s, int64_t request, int64_t *times) {
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->requests.find(request);
    if (it == s->requests.end()) return sfail(SVPF_EINVAL, "unknown request");
    Request *r = it->second.get();
    s->done_cv.wait(lk, [&] { return r->done; });
    if (times) { times[0] = r->arrival_ns; times[1] = r->admit_ns; times[2] = r->done_ns; }
    const int st = r->status;
    s->requests.erase(it);
    if (st == kCancelled) return sfail(SVPF_ECANCELED, "request cancelled before it was admitted");
    if (st < 0) return sfail(SVPF_EINVAL, "server shut down before the request started");
    if (st & 1) return sfail(SVPF_EPANIC, "SVAnalyse: the reference indexes out of range on this input (it panics)");
    if (st == 4) return sfail(SVPF_ECUDA, "enqueueing the request failed");
    if (st) return sfail(SVPF_EUNSUP, "SVAnalyse: unsupported input on the device path");
    return SVPF_OK;
}

int svpf_server_cancel(svpf_server *s, int64_t request) {
    if (!s) return sfail(SVPF_EINVAL, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->requests.find(request);
    if (it == s->requests.end()) return sfail(SVPF_EINVAL, "unknown request");
    Request *r = it->second.get();
    for (auto p = s->pending.begin(); p != s->pending.end(); ++p) {
        if (*p != r) continue;
        s->pending.erase(p);
        r->status = kCancelled;
        r->done = true;
        r->done_ns = s->now_ns();
        s->cancelled++;
        s->done_cv.notify_all();
        s->cv.notify_all();  // the request behind it may fit now
        return SVPF_OK;
    }
    return sfail(SVPF_EINVAL, r->done ? "request already finished" : "request already admitted: it runs to completion");
}

int64_t svpf_server_now_ns(const svpf_server *s) { return s->now_ns(); }

void svpf_server_stats(svpf_server *s, int64_t *admitted, int64_t *completed, int64_t *peak_device_bytes,
                       int32_t *peak_active, int64_t *kernel_launches) {
    std::lock_guard<std::mutex> lk(s->mu);
    if (admitted) *admitted = s->admitted;
    if (completed) *completed = s->completed;
    if (peak_device_bytes) *peak_device_bytes = s->peak_used;
    if (peak_active) *peak_active = s->peak_active;
    if (kernel_launches) *kernel_launches = s->launches.load();
}

void svpf_server_destroy(svpf_server *s) {
    if (!s) return;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        s->stopping = true;
        s->cv.notify_all();
    }
    s->worker.join();
    {
        std::unique_lock<std::mutex> lk(s->mu);
        s->done_cv.wait(lk, [&] { return s->active == 0; });
    }
    for (auto &st : s->streams) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    for (auto &ev : s->events)
        if (ev) cudaEventDestroy(ev);
    for (uint8_t *p : s->stage)
        if (p) cudaFreeHost(p);
    for (uint8_t *p : s->retired) cudaFreeHost(p);
    if (s->slot_status) cudaFreeHost(s->slot_status);
    delete s;
}

}  // extern "C"
