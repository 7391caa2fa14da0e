// noalloc.cu -- Analyse over a clip without any device allocation.
//
// Some callers cannot call cudaMalloc: a frame server's per-frame callback, where a
// device allocation can synchronise the whole device and stall every other filter's
// stream, or a host application that hands this library a fixed memory budget and
// forbids allocations once it is running. For them, svpf_clip_analyse_device_noalloc
// runs the Analyse kernel with its scratch in the fixed array below instead of a
// caller-provided buffer.
//
// The array is a file-scope device variable: every GPU that loads this library holds
// its kNoAllocScratchBytes until the process exits. Host code cannot use the array's
// name as a device address, so every call looks the address up with
// cudaGetSymbolAddress on the current device (cheap once the module is loaded, and
// never stale: a device reset or a new primary context gives the array a new address,
// which the next call picks up). All calls share the one array and it keeps what the
// last call left there: the status word is cleared on every call, and the search itself
// writes every scratch word before reading it. Two calls whose kernels overlap on the
// GPU (different streams, no ordering between them) race on the array and give
// undefined results; order them on one stream. Each call reads the kernel's status back
// into host memory and synchronises its stream, so it cannot be made on a stream that is
// being captured into a CUDA graph.
#include <cuda_runtime.h>

#include <string>

#include "../../include/svpflow_b200.h"
#include "handles.h"
#include "svpf_device.h"

namespace {

constexpr size_t kNoAllocScratchBytes = 32u << 20;  // 32 MiB
constexpr size_t kStatusBytes = 256;                // status word at the head of the array

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

}  // namespace

namespace {

int noalloc_fail(int code, const std::string &msg) {
    svpf::set_last_error(msg);
    return code;
}

// The device address of g_noalloc_scratch in the current device's context, looked up
// on every call (nothing is cached across calls, so no address outlives its context).
int scratch_address(unsigned char **out) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
        return noalloc_fail(SVPF_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    *out = (unsigned char *)p;
    return SVPF_OK;
}

}  // namespace

extern "C" int svpf_clip_analyse_device_noalloc(const svpf_analyser *a, const uint8_t *supers_dev, int32_t nframes,
                                                int32_t first, int32_t count, uint8_t *payloads_dev, void *stream) {
    using namespace svpf;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return noalloc_fail(SVPF_ECUDA, "no CUDA device: the svpflow_b200 library computes on an NVIDIA GPU only");
    if (!a) return noalloc_fail(SVPF_EINVAL, "null analyser");
    if (count <= 0) return SVPF_OK;
    if (first < 0 || first + count > nframes || !supers_dev || !payloads_dev)
        return noalloc_fail(SVPF_EINVAL, "bad frame range or buffers");
    const AnalyseParams &P = *analyser_params(a);
    if ((uintptr_t)payloads_dev & 3) return noalloc_fail(SVPF_EINVAL, "payloads must be 4-byte aligned");
    if (P.px_bytes == 2 && ((uintptr_t)supers_dev & 1))
        return noalloc_fail(SVPF_EINVAL, "16-bit super frames must be 2-byte aligned");
    const size_t need = kStatusBytes + (size_t)count * (size_t)P.scratch_per_pair;
    if (need > kNoAllocScratchBytes)
        return noalloc_fail(SVPF_EINVAL, "svpf_clip_analyse_device_noalloc: " + std::to_string(count) +
                                             " pairs need " + std::to_string(need) + " scratch bytes, above the " +
                                             std::to_string(kNoAllocScratchBytes) +
                                             "-byte static scratch; pass fewer pairs per call");
    unsigned char *scr = nullptr;
    if (int rc = scratch_address(&scr)) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(scr, 0, kStatusBytes, st);  // the status word must start at zero
    if (e != cudaSuccess) return noalloc_fail(SVPF_ECUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
    PairSrc src{};
    src.clip = supers_dev;
    src.frame_bytes = analyser_layout(a)->frame_bytes;
    src.first = first;
    src.nframes = nframes;
    const int32_t d = analyser_delta(a);
    src.delta = d > 1 ? d : 1;
    int nl = 0;
    e = launch_analyse(P, src, count, payloads_dev, scr + kStatusBytes, (int *)scr, st, &nl);
    add_launches(nl);
    if (e != cudaSuccess) return noalloc_fail(SVPF_ECUDA, std::string("analyse launch: ") + cudaGetErrorString(e));
    int status = 0;
    e = cudaMemcpyAsync(&status, scr, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return noalloc_fail(SVPF_ECUDA, std::string("status read: ") + cudaGetErrorString(e));
    if (status & 1) return noalloc_fail(SVPF_EPANIC, "SVAnalyse: the reference indexes out of range on this input (it panics)");
    if (status) return noalloc_fail(SVPF_EUNSUP, "SVAnalyse: unsupported input on the device path");
    return SVPF_OK;
}
