// svpf_device.h -- launch-side declarations shared by the CUDA translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "svpf_internal.h"

namespace svpf {

// Everything the Super kernels need about one (options, layout, source pitch) triple.
struct SuperDev {
    int32_t width, height, pel, levels, full, gpu, scale_up, scale_down;
    int32_t px_bytes, px_max;                 // sample size (1, 2) and largest sample (255, 1023)
    int64_t y_stride, c_stride, y_rows, c_rows, y_len, c_len;   // in samples
    int64_t frame_bytes;                      // bytes between super frames
    int64_t src_y_stride, src_c_stride, src_y_len, src_c_len;   // in samples
    int64_t src_frame_bytes;                  // bytes between source frames
    int32_t lw[kMaxLevels], lh[kMaxLevels];   // reduce_dim(luma_w/h, level)
    int64_t row_y[kMaxLevels], row_c[kMaxLevels];  // first row of each level in Y / chroma
};

bool make_super_dev(const SuperOpts &so, const SuperLayout &L, int64_t src_y_stride, int64_t src_c_stride,
                    SuperDev &D);
// src: nframes source frames (Y|U|V at src pitches, src_frame_bytes apart);
// dst: nframes super frames (frame_bytes apart). Adds its kernel launches to *launches.
cudaError_t launch_super(const SuperDev &D, const uint8_t *src, uint8_t *dst, int nframes, cudaStream_t stream,
                         int *launches);

// One frame pair of an Analyse launch: super frames of the current and reference frame.
struct PairRef {
    const uint8_t *cur;
    const uint8_t *ref;
};

// Where the pairs of a launch come from: an explicit device table, or a clip of
// contiguous super frames where pair b is (first + b, min(first + b + delta, nframes - 1)).
struct PairSrc {
    const PairRef *table;
    const uint8_t *clip;
    int64_t frame_bytes;
    int32_t first, nframes, delta;
    unsigned long long *stats;  // nullable: level-0 look-ahead counters (see search_level0_spec)
};

// One work item of a batch launch: a frame pair of some clip and where its payload goes.
struct BatchItem {
    PairRef pair;
    uint8_t *payload;
    int32_t clip;   // index into the launch's AnalyseParams table (and status array)
    int32_t pad_;
};

// The launchers every Analyse variant TU exports (analyse_body.cuh).
#define SVPF_DECLARE_ANALYSE_VARIANT(ns)                                                                          \
    namespace ns {                                                                                                \
    size_t dir_shared_bytes();                                                                                    \
    cudaError_t launch_plain(const AnalyseParams &P, const PairSrc &src, int npairs, uint8_t *payloads,           \
                             uint8_t *scratch, int *status_dev, cudaStream_t stream, int *launches);              \
    cudaError_t batch_blocks_per_sm(int *blocks);                                                                 \
    cudaError_t launch_batch(const AnalyseParams *clips_dev, const BatchItem *items_dev, int nitems,              \
                             unsigned *next_item_dev, uint8_t *scratch, int64_t scratch_per_cta,                  \
                             int *clip_status_dev, int grid, cudaStream_t stream, int *launches);                 \
    }
SVPF_DECLARE_ANALYSE_VARIANT(nt128)
SVPF_DECLARE_ANALYSE_VARIANT(nt64)
SVPF_DECLARE_ANALYSE_VARIANT(nt32)
SVPF_DECLARE_ANALYSE_VARIANT(nt128b3)
SVPF_DECLARE_ANALYSE_VARIANT(nt64b6)
SVPF_DECLARE_ANALYSE_VARIANT(nt128p16)  // uint16 samples (AnalyseParams::px_bytes == 2)


// A compiled launch shape of the Analyse kernels: threads per search direction and the
// resident CTAs per SM its register budget was cut for. Results do not depend on it.
struct AnalyseVariant {
    const char *name;
    int threads_per_dir, min_blocks;
    cudaError_t (*launch_plain)(const AnalyseParams &, const PairSrc &, int, uint8_t *, uint8_t *, int *,
                                cudaStream_t, int *);
    cudaError_t (*batch_blocks_per_sm)(int *);
    cudaError_t (*launch_batch)(const AnalyseParams *, const BatchItem *, int, unsigned *, uint8_t *, int64_t, int *,
                                int, cudaStream_t, int *);
};
int analyse_variant_count();
const AnalyseVariant &analyse_variant(int i);  // 0 = the plain path's default (nt128)

// Analyse over npairs pairs with the default variant; payloads npairs x P.payload_len
// bytes, scratch npairs x P.scratch_per_pair bytes, status one int (0 = ok), cleared by
// the caller.
cudaError_t launch_analyse(const AnalyseParams &P, const PairSrc &src, int npairs, uint8_t *payloads,
                           uint8_t *scratch, int *status_dev, cudaStream_t stream, int *launches);
// The same with a given launch shape (analyse_variant index).
cudaError_t launch_analyse_shape(int variant, const AnalyseParams &P, const PairSrc &src, int npairs, uint8_t *payloads,
                                 uint8_t *scratch, int *status_dev, cudaStream_t stream, int *launches);
// The shape of the server's chunk launches, which share the GPU with other clips' chunks: nt128,
// whose level 0 spreads over the SMs (measured at 5 clips/s against nt128_b3: 83.0 against 60.4
// pairs/s, p50 7.9 against 13.1 s, p99 25.7 against 36.5 s).
constexpr int kShapeShared = 0;

}  // namespace svpf
