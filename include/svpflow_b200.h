/*
 * svpflow_b200.h -- C ABI of the B200 motion-analysis library (libsvpflow_b200.so).
 *
 * Drop-in for open-svpflow's svpflow1 motion-analysis path: the Super pyramid builder
 * and the Analyse block search, computed on an NVIDIA B200 (sm_100a), byte-identical to
 * the reference's CPU output. Plain pointers and sizes only. Each entry point names the
 * reference interface it replaces (paths inside the reference project).
 *
 * Buffers
 *   source frame  packed I420/YUV420P8: Y (w*h) | U (w/2*h/2) | V (w/2*h/2)
 *   super frame   Y (w * H) | U (w/2 * H/2) | V (w/2 * H/2), H = svpf_super_height();
 *                 the layout of crates/svpflow1/src/portable.rs:104-106 (SuperFrame::bytes)
 *   payload       the Analyse output frame row: crates/svpflow1/src/analyse_search.rs:2740-2811
 * Functions returning int return 0 on success, else a negative code; the message is in
 * svpf_last_error() (thread-local). Handles are immutable after creation; the host-buffer
 * entry points of one analyser serialise on an internal lock, the device entry points
 * take caller-owned buffers and a cudaStream_t (passed as void*) and never allocate.
 */
#ifndef SVPFLOW_B200_H
#define SVPFLOW_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct svpf_super svpf_super;
typedef struct svpf_analyser svpf_analyser;

#define SVPF_OK 0
#define SVPF_EINVAL (-1)   /* bad argument or option (message as the reference's setError text) */
#define SVPF_ECUDA (-2)    /* CUDA runtime error or no usable device */
#define SVPF_EPANIC (-3)   /* input on which the reference indexes out of range (it would panic) */
#define SVPF_EUNSUP (-4)   /* option combination not available on the device path */
#define SVPF_ECANCELED (-5) /* served request cancelled before it was admitted (svpf_server_cancel) */

/* Thread-local text of the last error. */
const char *svpf_last_error(void);
/* Library version of the reference plugin this replaces: svpGetVersion(),
 * crates/svpflow1/src/abi.rs:3-9 (1174405393). */
int64_t svpf_reference_version(void);

/* ---------------------------------------------------------------- Super */
/* Super filter creation: SuperOpts::from_opt + pack_data + super_height
 * (crates/svpflow1/src/super_opts.rs:17-95, super_filter.rs:67-82). `opt` is the
 * VapourSynth `opt:data` string (lenient JSON, crates/svpflow-core/src/params.rs);
 * NULL or an unparsable string means defaults, as in super_filter.rs:107-121. */
int svpf_super_create(int32_t width, int32_t height, const char *opt, size_t opt_len, svpf_super **out);
/* svpf_super_create for `bits` = 8 (identical) or 10: this project's 10-bit extension, which
 * the reference does not have (it is 8-bit only). Frames are then uint16 samples 0..1023,
 * every size and offset of the API counts samples except the *_len / buffer sizes, which are
 * bytes; the Super arithmetic is the same with its clamps at 1023. */
int svpf_super_create_bits(int32_t width, int32_t height, const char *opt, size_t opt_len, int32_t bits,
                           svpf_super **out);
int32_t svpf_super_bits(const svpf_super *s);
/* SuperBuilder::new(width, height, pel) (crates/svpflow1/src/portable.rs:30-62). */
int svpf_super_create_portable(int32_t width, int32_t height, int32_t pel, svpf_super **out);
void svpf_super_destroy(svpf_super *s);
int64_t svpf_super_sdata(const svpf_super *s);       /* SuperOpts::pack_data, super_opts.rs:51-63 */
int32_t svpf_super_height(const svpf_super *s);      /* SuperOpts::super_height, super_opts.rs:65-67 */
int32_t svpf_super_levels(const svpf_super *s);      /* SuperBuilder::levels, portable.rs:79-82 */
int32_t svpf_super_pel(const svpf_super *s);
size_t svpf_super_source_len(const svpf_super *s);   /* SuperBuilder::source_len, portable.rs:84-87 */
size_t svpf_super_output_len(const svpf_super *s);   /* SuperBuilder::output_len, portable.rs:89-92 */
/* SuperBuilder::build (portable.rs:94-148) / get_frame_super (super_filter.rs:143-268)
 * over nframes frames, host buffers in and out. */
int svpf_super_build(const svpf_super *s, const uint8_t *src, uint8_t *dst, int32_t nframes);
/* Same on device buffers: nframes source frames at `src_pitch`-strided planes
 * (src_y_stride / src_c_stride samples per row; 0 = packed) -> nframes super frames. */
int svpf_super_build_device(const svpf_super *s, const uint8_t *src_dev, int64_t src_y_stride,
                            int64_t src_c_stride, uint8_t *dst_dev, int32_t nframes, void *stream);

/* ---------------------------------------------------------------- Analyse */
/* Analyse filter creation: AnalyseOpts::from_opt with the super clip's `sdata`
 * (crates/svpflow1/src/analyse_opts.rs:45-219, analyse_filter.rs:84-101); src_width /
 * src_height (> 0) override the frame size as analyse_filter.rs:96-101 does. */
int svpf_analyser_create(int64_t sdata, const char *opt, size_t opt_len, int32_t src_width,
                         int32_t src_height, svpf_analyser **out);
/* svpf_analyser_create over super frames of `bits` = 8 or 10 (uint16 samples; the 10-bit
 * extension: chroma default 512 on clamped reads, payload luma byte = block mean >> 2, all
 * else as for 8 bits). Batches and the server take 8-bit clips only. */
int svpf_analyser_create_bits(int64_t sdata, const char *opt, size_t opt_len, int32_t src_width,
                              int32_t src_height, int32_t bits, svpf_analyser **out);
/* Analyser::new(super_builder, block w, block h, overlap mode, vectors)
 * (crates/svpflow1/src/portable.rs:189-229). */
int svpf_analyser_create_portable(const svpf_super *s, int32_t block_w, int32_t block_h,
                                  int32_t overlap_mode, int32_t vectors, svpf_analyser **out);
void svpf_analyser_destroy(svpf_analyser *a);
/* The 16-int vector header whose address the reference publishes as `vdata`
 * (pack_vdata_header, analyse_search.rs:2813-2841; Analyser::vector_header,
 * portable.rs:231-234). Valid for the analyser's lifetime. */
const int32_t *svpf_analyser_vdata(const svpf_analyser *a);
/* Bytes of one Analyse output frame (analyse_filter.rs:122-129). */
size_t svpf_analyser_payload_len(const svpf_analyser *a);
int32_t svpf_analyser_delta(const svpf_analyser *a);
/* Device scratch the *_device entry points need for `npairs` concurrent pairs. */
size_t svpf_analyser_scratch_bytes(const svpf_analyser *a, int32_t npairs);
/* Analyser::analyse(current, reference) (portable.rs:236-250) on host super frames. */
int svpf_analyse(svpf_analyser *a, const uint8_t *cur_super, const uint8_t *ref_super, uint8_t *payload);
/* analyse_pair + pack_vector_frame for npairs pairs of device super frames:
 * cur_dev[i] / ref_dev[i] are device pointers (host arrays of them), payloads_dev holds
 * npairs * payload_len bytes, scratch_dev svpf_analyser_scratch_bytes(npairs). */
int svpf_analyse_pairs_device(const svpf_analyser *a, const uint8_t *const *cur_dev,
                              const uint8_t *const *ref_dev, int32_t npairs, uint8_t *payloads_dev,
                              void *scratch_dev, void *stream);
/* A clip as the VapourSynth Analyse filter sees it: output frame n pairs super frame n
 * with super frame min(n + delta, nframes - 1) (analyse_filter.rs:240-282). Frames
 * [first, first + count) of `supers_dev` (nframes contiguous super frames) -> payloads. */
int svpf_clip_analyse_device(const svpf_analyser *a, const uint8_t *supers_dev, int32_t nframes,
                             int32_t first, int32_t count, uint8_t *payloads_dev, void *scratch_dev,
                             void *stream);
/* Status of the last device launch that used `scratch_dev` (synchronises `stream`):
 * SVPF_OK, or SVPF_EPANIC when a pair hit an input the reference cannot process. */
int svpf_device_status(const void *scratch_dev, void *stream);
/* No counterpart in the reference (a tuning knob). Level 0 runs with look-ahead by default:
 * each warp of a search direction takes its own block in the reference's order, searches it
 * without the neighbour vectors not yet committed, then, in order, re-checks the reference's
 * selection with them and repeats the refinement when one wins; results are bit-identical
 * with it on or off. `levels` is a bit set: 1 level 0, 2 the coarser levels, 4 level 0 spread
 * over the GPU (with 1: a launch of its own with one CTA per warp, so every SM carries the same
 * share of the walking warps; the pair kernel and a finish kernel run before and after it).
 * 0 turns it off; the default is 5. Only the 128-thread launch shape with two CTAs per SM runs
 * it (the plain path's shape for launches of at most two frame pairs per SM); the others always
 * keep the serial order. Affects launches made after the call. */
int svpf_analyser_set_lookahead(svpf_analyser *a, int32_t levels);
/* The look-ahead counters of the last device launch on `scratch_dev` (synchronises `stream`):
 * out[0] level-0 blocks, out[1] blocks with deferred neighbour seeds, out[2] deferred seeds
 * evaluated, out[3] refinements run again. */
int svpf_device_lookahead_stats(const void *scratch_dev, void *stream, int64_t out[4]);
/* No counterpart in the reference. The same Analyse over a clip as
 * svpf_clip_analyse_device, for callers that cannot allocate device memory (a frame
 * server's per-frame callback, where cudaMalloc can synchronise the device and stall other
 * streams, or a host that forbids allocations after start-up): the kernel's scratch is a
 * fixed 32 MiB array inside this library (every GPU that loads the library holds it until
 * exit), so no scratch argument is taken and nothing is allocated. Returns SVPF_EINVAL when
 * `count` pairs need more than that array (use fewer pairs per call). Every call looks the
 * array's device address up in the current context. Calls share the array: calls whose
 * kernels overlap on the GPU race, so order them on one stream. Synchronises `stream` and
 * returns the kernel's status (SVPF_OK, SVPF_EPANIC); because it synchronises, it must not
 * be called on a stream that is being captured into a CUDA graph. */
int svpf_clip_analyse_device_noalloc(const svpf_analyser *a, const uint8_t *supers_dev, int32_t nframes,
                                     int32_t first, int32_t count, uint8_t *payloads_dev, void *stream);
/* Whole clip from host source frames: Super over every frame, then Analyse for output
 * frames [first, first + count); payloads = count * payload_len host bytes. */
int svpf_clip_analyse(svpf_analyser *a, const svpf_super *s, const uint8_t *frames, int32_t nframes,
                      int32_t first, int32_t count, uint8_t *payloads);

/* Number of kernels this thread launched through the library since the last reset. */
int64_t svpf_kernel_launches(void);
void svpf_kernel_launches_reset(void);

/* ---------------------------------------------------------------- payload consumers */
/* The motion-vector grid a frame interpolator samples for a vdata header: metadata.rs
 * vector_data (:89-115) and motion_grid / extended_grid (crates/svpflow-core/src/metadata.rs:211-244). */
int svpf_vector_grid(const int32_t *vdata, int32_t *motion_w, int32_t *motion_h);
/* decode_vectors (crates/svpflow-core/src/metadata.rs:246-273) and vector_planes
 * (crates/svpflow-core/src/renderer.rs:1680-1726) as SmoothFps applies them (svpflow2 core.rs:962-1001),
 * on the device: `npayloads` Analyse payloads (payload_len bytes apart) -> per payload four uint16
 * planes mvx0 | mvy0 | mvx1 | mvy1 of motion_w x motion_h (centred on 1024; 0 = previous set,
 * 1 = current set), vectors clamped to the frame_w x frame_h frame unless `raw`. status_dev[i]
 * becomes 1 where payload i does not decode (the reference's None). Asynchronous on `stream`. */
int svpf_vector_planes_device(const int32_t *vdata, const uint8_t *payloads_dev, size_t payload_len, int32_t npayloads,
                              int32_t frame_w, int32_t frame_h, int32_t raw, uint16_t *planes_dev, int32_t *status_dev,
                              void *stream);
/* SmoothFps' mask planes for the frame it interpolates at `phase` (0..256) between a payload's two
 * frames (svpflow2 core.rs:1154-1195, :1467-1499, :1605-1616): per payload five byte planes of
 * motion_w x motion_h, cover0 | cover1 | area0 | area1 | area_max. cover0 / cover1 = coverage_mask
 * (crates/svpflow-core/src/renderer.rs:1738-1763) of the current set at 256 - phase and of the
 * previous set at phase, `cover_percent` strong (the mask.cover option); area0 / area1 =
 * magnitude_mask (:1647-1678) of the previous / current set with area_scale and area_sharp (the
 * mask.area options); area_max = max_mask (:2908-2915) of the two. cover0, cover1 are the masks
 * svpf_render_masked_device / svpf_render_mode23_device take and area_max their final mask; area0,
 * area1 are the masks of svpf_render_blend_device, and area0 (algorithm 1) or area1 (algorithm 2)
 * the mask of svpf_render_warp_device. scratch_dev holds svpf_render_masks_scratch bytes.
 * Payloads (payload_len a multiple of 4) and scratch are 4-byte aligned; the overlap lies in
 * 0..block - 1 and grid_w * grid_h * block area <= 2^30 (every Analyse field). status_dev[i] = 1
 * where payload i does not decode (its planes are left as they were). Bytes equal the reference's
 * for area_sharp >= 0.001 and area_scale >= 0 (the magnitude byte's steps are found on the host with
 * libm's pow); other settings evaluate pow on the device (CUDA's, within 2 ulp of libm's).
 * Asynchronous on `stream`. */
int64_t svpf_render_masks_scratch(const int32_t *vdata, int32_t npayloads); /* -1 (and svpf_last_error) if refused */
int svpf_render_masks_device(const int32_t *vdata, const uint8_t *payloads_dev, size_t payload_len, int32_t npayloads,
                             int32_t phase, int32_t cover_percent, double area_scale, double area_sharp,
                             uint8_t *masks_dev, void *scratch_dev, int32_t *status_dev, void *stream);

/* SmoothFps's scene limits (svpflow2 options.rs SceneLimits; SmoothFps's defaults: blocks 20, zero
 * 200, m1 1600, m2 2800, scene 4000), as metadata.rs SceneThresholds reads them. */
typedef struct {
    int32_t blocks_pct, zero, m1, m2, scene;
} svpf_scene_limits;
/* SmoothFps's scene class (0 steady .. 3 scene change) of each payload (svpflow2 core.rs:2079-2100:
 * metadata.rs analyze_scene, crates/svpflow-core/src/metadata.rs:349-361, over the previous and
 * current sets, each falling back to the other; 3 when the payload holds neither), with the
 * scene.luma gamma (default 1.5). classes_dev[i] = -1 and status_dev[i] = 1 where payload i does not
 * decode. Payloads (payload_len a multiple of 4) are 4-byte aligned. Bit-exact: the luma curve is
 * tabulated on the host with libm's pow. Asynchronous on `stream`. */
int svpf_scene_class_device(const int32_t *vdata, const uint8_t *payloads_dev, size_t payload_len, int32_t npayloads,
                            double luma_gamma, const svpf_scene_limits *limits, int32_t *classes_dev,
                            int32_t *status_dev, void *stream);

/* ---------------------------------------------------------------- frame render (SmoothFps) */
/* renderer.rs CpuConfig (crates/svpflow-core/src/renderer.rs:34-46) as SmoothFps fills it
 * (svpflow2 core.rs:1501-1517); chroma is 4:2:0. */
typedef struct {
    int32_t width, height;        /* frame size */
    int32_t block_w, block_h;     /* the vectors' effective block: block - overlap (vdata[2] - vdata[9], vdata[3] - vdata[10]) */
    int32_t origin_x, origin_y;   /* vdata block / 2 */
    int32_t grid_w, grid_h;       /* motion-plane size (svpf_vector_grid) */
    int32_t source_step;          /* 1 for frames; the super clip's pel when the sources are super frames */
} svpf_render_config;
/* CpuRenderer::render_mode1_or_2 (renderer.rs:308-328, render_selected_warp_rows :876-984) on
 * the device: the three planes of one output frame, each sample the source sample displaced by the
 * motion of (motion_x, motion_y) (uint16 planes of grid_w x grid_h, as svpf_vector_planes_device
 * writes them) scaled by the threshold LUT (set_threshold :238-250, threshold 0..256): mode1 != 0
 * uses the inverse LUT (256 - threshold) and the caller passes the second source and motion set,
 * mode 2 the threshold LUT with the first, as render_mode1_or_2 does. interp: bilinear motion
 * between the four block centres (else one motion per block). mask: NULL, or the mode's mask
 * plane (grid_w x grid_h bytes; masks.a for mode 1, masks.b for mode 2): each sample is then
 * mode1_pixel(undisplaced, displaced, alpha) with alpha interpolated from the mask (:1818-1820).
 * src_shift 0: src[] are plain planes (stride bytes per row); log2(source_step): src[] are a
 * super clip's level-0 planes whose sub-planes lie stride x plane-height bytes apart (svpflow2
 * core.rs:3340-3388); src_len bounds every read. dst[p] must hold the plane's rows (height, or
 * height / 2 for chroma) of dst_stride[p] >= width bytes; motion (and mask) planes hold grid_w x
 * grid_h entries. Device pointers; asynchronous on `stream`. */
int svpf_render_warp_device(const svpf_render_config *cfg, int32_t threshold, int32_t mode1, int32_t interp,
                            const uint8_t *const src[3], const int64_t src_stride[3], const int64_t src_len[3],
                            int32_t src_shift, const uint16_t *motion_x, const uint16_t *motion_y,
                            const uint8_t *mask, uint8_t *const dst[3], const int64_t dst_stride[3], void *stream);
/* CpuRenderer::render_mode11_or_13 (renderer.rs:330-438; zero_origin != 0: its zero-origin variant
 * :356-380) on the device: each sample blends source 0 displaced by motion set 0 (threshold LUT)
 * with source 1 displaced by motion set 1 (inverse LUT): mode 11 blend_256(mv0, mv1, threshold),
 * mode 13 (mode13 != 0) blend_256(cur0, cur1, threshold) clamped between mv0 and mv1
 * (mode11_or_13_pixel :2918-2943). mask_a / mask_b: both NULL, or the two masks whose max_mask
 * blends the result with the undisplaced blend. Sources, strides and src_shift as for
 * svpf_render_warp_device; device pointers; asynchronous on `stream`. */
int svpf_render_blend_device(const svpf_render_config *cfg, int32_t threshold, int32_t mode13, int32_t interp,
                             int32_t zero_origin, const uint8_t *const src0[3], const int64_t src0_stride[3],
                             const int64_t src0_len[3], const uint8_t *const src1[3], const int64_t src1_stride[3],
                             const int64_t src1_len[3], int32_t src_shift, const uint16_t *motion0_x,
                             const uint16_t *motion0_y, const uint16_t *motion1_x, const uint16_t *motion1_y,
                             const uint8_t *mask_a, const uint8_t *mask_b, uint8_t *const dst[3],
                             const int64_t dst_stride[3], void *stream);
/* CpuRenderer::render_mode21_or_22 (renderer.rs:571-641) on the device: the reads of
 * svpf_render_blend_device, each pair of displaced samples blended by the alphas of mask_a and mask_b
 * (both required): mode 21 blend_256(blend_255(mv0, mv1, a0), blend_255(mv1, mv0, a1), threshold),
 * mode 22 (mode22 != 0) blend_256(cur0, cur1, threshold) clamped between those two (mode21_pixel /
 * mode22_pixel :1830-1848); final_mask (optional) blends the result towards blend_256(cur0, cur1,
 * threshold_limit), threshold_limit from the threshold and mask_scale as set_threshold_value (:256-264)
 * computes it. No interpolation (interp == 0) puts the grid at zero origin, as the reference does. */
int svpf_render_masked_device(const svpf_render_config *cfg, int32_t threshold, double mask_scale, int32_t mode22,
                              int32_t interp, const uint8_t *const src0[3], const int64_t src0_stride[3],
                              const int64_t src0_len[3], const uint8_t *const src1[3], const int64_t src1_stride[3],
                              const int64_t src1_len[3], int32_t src_shift, const uint16_t *motion0_x,
                              const uint16_t *motion0_y, const uint16_t *motion1_x, const uint16_t *motion1_y,
                              const uint8_t *mask_a, const uint8_t *mask_b, const uint8_t *final_mask,
                              uint8_t *const dst[3], const int64_t dst_stride[3], void *stream);
/* CpuRenderer::render_mode23 (renderer.rs:644-666, render_mode23_plane_rows_inner :1294-1537) on the
 * device: four motion sets motion_x/y[0..3] = base0, base1, next0, prev1 (sets 0 and 2 read source 0
 * with the threshold LUT, 1 and 3 source 1 with the inverse LUT); mode23_pixel (:1850-1868) with
 * alphas from mask_a and mask_b (required) and final_mask (optional) blending towards
 * blend_256(cur0, cur1, threshold). Zero origin when interp == 0, as the reference. */
int svpf_render_mode23_device(const svpf_render_config *cfg, int32_t threshold, int32_t interp,
                              const uint8_t *const src0[3], const int64_t src0_stride[3], const int64_t src0_len[3],
                              const uint8_t *const src1[3], const int64_t src1_stride[3], const int64_t src1_len[3],
                              int32_t src_shift, const uint16_t *const motion_x[4], const uint16_t *const motion_y[4],
                              const uint8_t *mask_a, const uint8_t *mask_b, const uint8_t *final_mask,
                              uint8_t *const dst[3], const int64_t dst_stride[3], void *stream);

/* ---------------------------------------------------------------- batched form */
/* No counterpart in the reference, which analyses one clip at a time, one output frame
 * per getFrame call (crates/svpflow1/src/analyse_filter.rs:229-334). A batch holds many
 * clips of any size and length (each with its own Super and Analyse handles, as for
 * svpf_clip_analyse) and analyses every output frame of every clip in one persistent
 * launch replayed from a CUDA graph; each payload is byte-identical to the per-clip
 * call's. Creation allocates all device memory of the batch (svpf_batch_device_bytes):
 * the clips' source frames, super frames and payloads plus the work list and scratch.
 * A batch serialises its own calls. */
typedef struct svpf_batch svpf_batch;
int svpf_batch_create(int32_t nclips, const svpf_super *const *supers, const svpf_analyser *const *analysers,
                      const int32_t *nframes, svpf_batch **out);
void svpf_batch_destroy(svpf_batch *b);
int32_t svpf_batch_clips(const svpf_batch *b);
int64_t svpf_batch_pairs(const svpf_batch *b);           /* output frames over all clips */
size_t svpf_batch_device_bytes(const svpf_batch *b);
/* Device address of clip `clip`'s source frames (nframes packed I420 frames, in order),
 * for callers that fill them on the device; NULL for a bad index. */
uint8_t *svpf_batch_frames_device(svpf_batch *b, int32_t clip);
/* Device address of clip `clip`'s payloads (nframes x payload_len bytes). */
const uint8_t *svpf_batch_payloads_device(const svpf_batch *b, int32_t clip);
/* Host buffers in and out: copies every clip's frames in, runs, copies every payload
 * out, synchronises and returns the first failing clip's status. */
int svpf_batch_run(svpf_batch *b, const uint8_t *const *frames, uint8_t *const *payloads);
/* Device-resident form: replays the run on `stream` over the frames already in place;
 * NULL means the batch's own stream, not the legacy default stream. svpf_batch_status
 * synchronises that stream and reports. */
int svpf_batch_launch(svpf_batch *b, void *stream);
int svpf_batch_status(svpf_batch *b, void *stream);
/* Launch shape: compiled variant (threads per search direction, see
 * svpf_analyse_variant_name) and 4x4 tiles per lane (2, 4 or 8). Results do not depend
 * on it. svpf_batch_autotune times the shapes on the batch's largest pairs (frames must be
 * in place), keeps the fastest and remembers it per device and clip mix (and in the file
 * named by the SVPF_TUNE_CACHE environment variable, when set). */
int svpf_batch_set_shape(svpf_batch *b, int32_t variant, int32_t tiles_per_lane);
const char *svpf_batch_shape(const svpf_batch *b, int32_t *variant, int32_t *tiles_per_lane, int32_t *grid);
int svpf_batch_autotune(svpf_batch *b, int32_t *variant, int32_t *tiles_per_lane, double *pairs_per_s);
int32_t svpf_batch_graph_launches(const svpf_batch *b);  /* kernels in one replay */
int32_t svpf_analyse_variant_count(void);
const char *svpf_analyse_variant_name(int32_t i);

/* ---------------------------------------------------------------- served form */
/* No counterpart in the reference. A server analyses clips that arrive over time with
 * continuous batching: a scheduler thread admits submitted clips in arrival order while
 * their device memory fits `hbm_budget_bytes` and fewer than `max_active` clips are in
 * flight; each admitted clip runs on its own stream (frames in, Super, Analyse in chunks
 * of `chunk_pairs` output frames, each chunk's payloads out as it completes), overlapping
 * on the device with the others. Payloads are byte-identical to svpf_clip_analyse's. */
typedef struct svpf_server svpf_server;
int svpf_server_create(size_t hbm_budget_bytes, int32_t max_active, int32_t chunk_pairs, svpf_server **out);
/* Stops admitting, waits for the admitted clips; clips never admitted fail. */
void svpf_server_destroy(svpf_server *s);
/* Queues a clip: `frames` (nframes packed I420 frames) and `payloads` (nframes x
 * payload_len bytes) are host buffers that must stay valid until svpf_server_wait
 * returns (pinned memory lets the copies run asynchronously). When `pair_done_ns` is
 * given (nframes entries), entry n receives the server-clock time at which payload n
 * reached host memory. The Super and Analyse handles must outlive the request. */
int svpf_server_submit(svpf_server *s, const svpf_super *sup, const svpf_analyser *an, const uint8_t *frames,
                       int32_t nframes, uint8_t *payloads, int64_t *pair_done_ns, int64_t *request);
/* Blocks until the request finished and returns its status; times[0..2] (optional)
 * receive its arrival, admission and completion times on the server clock. */
int svpf_server_wait(svpf_server *s, int64_t request, int64_t *times);
/* Withdraws a request that has not been admitted yet: it never runs, its buffers are no longer
 * used when this returns SVPF_OK, and svpf_server_wait on it returns SVPF_ECANCELED. A request
 * already admitted runs to completion (its work is queued on the device): SVPF_EINVAL, as for
 * an unknown or finished request. */
int svpf_server_cancel(svpf_server *s, int64_t request);
int64_t svpf_server_now_ns(const svpf_server *s);       /* the server clock, ns */
void svpf_server_stats(svpf_server *s, int64_t *admitted, int64_t *completed, int64_t *peak_device_bytes,
                       int32_t *peak_active, int64_t *kernel_launches);

#ifdef __cplusplus
}
#endif
#endif
