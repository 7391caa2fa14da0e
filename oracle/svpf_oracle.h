/*
 * svpf_oracle.h -- CPU restatement of open-svpflow's svpflow1 motion-analysis path
 * (Super pyramid + Analyse block search), used ONLY as a test checker.
 *
 * TEST INFRASTRUCTURE. Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / reference leg may load this library. The product (the CUDA
 * library under open-svpflow_b200/) never links or calls it.
 *
 * PARITY UNPINNED: the reference (Rust, crates/svpflow1) cannot be built in this
 * image (no cargo/rustc) and ships no tests, fixtures or golden vectors. This file
 * is a line-by-line restatement of the reference's scalar semantics; it is guarded
 * by an independent Python restatement (oracle/svpf_oracle_py.py) on small cases
 * and by primitive-level known-answer tests, not by reference outputs.
 *
 * All citations are paths inside the reference project.
 */
#ifndef SVPF_ORACLE_H
#define SVPF_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Sample type. The reference is 8-bit only; building with OR_PX16 gives this project's 10-bit
 * extension (uint16 samples 0..1023, chroma default 512, block luma byte = mean >> 2), which
 * has no reference behaviour and is checked against nothing but itself. */
#ifdef OR_PX16
typedef uint16_t or_px;
#else
typedef uint8_t or_px;
#endif

/* One looked-up option value: the result of Value::at(path) in
 * crates/svpflow-core/src/params.rs:69-85 (absent when the path does not exist). */
enum {
    OR_ABSENT = 0,
    OR_NUMBER = 1,
    OR_BOOL = 2,
    OR_NULL = 3,
    OR_STRING = 4,
    OR_ARRAY = 5,
    OR_OBJECT = 6
};

typedef struct {
    int32_t kind;     /* OR_* */
    int32_t nonempty; /* strings / arrays / objects: !is_empty() */
    double num;       /* OR_NUMBER: the parsed f64; OR_BOOL: 0 or 1 */
} or_val;

/* Key paths read by SuperOpts::from_opt (super_opts.rs:17-36) and
 * AnalyseOpts::from_opt (analyse_opts.rs:45-174). "refine0." means the first
 * element of the `refine` array (analyse_opts.rs:150-152). */
enum {
    OK_PEL = 0, OK_GPU, OK_SCALE_DOWN, OK_SCALE_UP, OK_FULL, OK_RC,
    OK_VECTORS, OK_BLOCK_W, OK_BLOCK_H, OK_BLOCK_OVERLAP, OK_SPECIAL_DELTA, OK_DELTA,
    OK_MAIN_PENALTY_LAMBDA, OK_PENALTY_LAMBDA,
    OK_MAIN_PENALTY_LSAD, OK_PENALTY_LSAD,
    OK_MAIN_PENALTY_PLEVEL, OK_PENALTY_PLEVEL,
    OK_MAIN_PENALTY_PNEW, OK_PENALTY_PNEW,
    OK_MAIN_PENALTY_PGLOBAL, OK_PENALTY_PGLOBAL,
    OK_MAIN_PENALTY_PZERO, OK_PENALTY_PZERO,
    OK_MAIN_PENALTY_PNBOUR, OK_PENALTY_PNBOUR,
    OK_MAIN_PENALTY_PREV, OK_PENALTY_PREV,
    OK_MAIN_SEARCH_TYPE, OK_SEARCH_TYPE,
    OK_MAIN_SEARCH_DISTANCE, OK_SEARCH_DISTANCE,
    OK_MAIN_SEARCH_COARSE_TYPE, OK_SEARCH_COARSE_TYPE,
    OK_MAIN_SEARCH_COARSE_DISTANCE, OK_SEARCH_COARSE_DISTANCE,
    OK_MAIN_SEARCH_COARSE_TRYMANY, OK_SEARCH_COARSE_TRYMANY,
    OK_MAIN_SEARCH_COARSE_BAD_SAD, OK_SEARCH_COARSE_BAD_SAD,
    OK_MAIN_SEARCH_COARSE_BAD_RANGE,
    OK_MAIN_SEARCH_SATD, OK_SEARCH_SATD,
    OK_MAIN_SEARCH_COARSE_SATD,
    OK_MAIN_SEARCH_SORT, OK_SORT,
    OK_REFINE0, /* the first element of `refine` itself (present or not) */
    OK_REFINE0_THSAD, OK_REFINE0_SEARCH_TYPE, OK_REFINE0_SEARCH_DISTANCE, OK_REFINE0_SEARCH_SATD,
    OK_MAIN_LEVELS,
    OK_COUNT
};

/* SuperOpts, super_opts.rs:3-14 */
typedef struct {
    int32_t pel, gpu, scale_down, scale_up;
    int32_t full, rc;
    int32_t levels, width, height;
} or_super_opts;

/* AnalyseOpts, analyse_opts.rs:4-42 */
typedef struct {
    int32_t vectors, block_w, block_h, overlap_mode, overlap_x, overlap_y, delta, pel, selector;
    int32_t levels, super_levels, width, height, lambda, lsad;
    double plevel;
    int32_t pnew, pglobal, pzero, pnbour, prev;
    int32_t search_type, coarse_search_type, distance, coarse_distance;
    int32_t coarse_trymany, coarse_bad_sad, coarse_bad_range;
    int32_t fine_satd, coarse_satd;
    int32_t has_refine_thsad, refine_thsad, refine_search_type, refine_distance, refine_satd;
    int32_t sort;
} or_analyse_opts;

/* Vec8, analyse_search.rs:25-31 */
typedef struct {
    int16_t dx, dy;
    uint32_t score;
    uint8_t luma;
    uint8_t pad_[3];
} or_vec8;

/* SuperPlanes, analyse_search.rs:33-46 (slices carry their lengths). */
typedef struct {
    const or_px *y; size_t y_len, y_stride;
    const or_px *u; size_t u_len, u_stride;
    const or_px *v; size_t v_len, v_stride;
    size_t luma_w, luma_h;
    int32_t pel, levels, full;
} or_planes;

/* ---- options ---- */
int or_super_opts_from_opt(const or_val *raw, int32_t width, int32_t height, or_super_opts *out,
                           char *err, size_t err_len);
int64_t or_super_pack_data(const or_super_opts *o);
int32_t or_super_height(const or_super_opts *o);
int32_t or_reduce_dim(int32_t dim, int32_t n);
int32_t or_auto_levels(int32_t width, int32_t height);
int32_t or_super_plane_height(int32_t base_h, int32_t pel, int32_t levels, int32_t full);
int or_analyse_opts_from_opt(const or_val *raw, int64_t sdata, const or_super_opts *hint,
                             or_analyse_opts *out, char *err, size_t err_len);
int or_overlap_from_mode(int32_t bw, int32_t bh, int32_t mode, int32_t *ox, int32_t *oy,
                         char *err, size_t err_len);
int32_t or_auto_search_levels(int32_t w, int32_t h, int32_t bw, int32_t bh, int32_t ox, int32_t oy);
/* Analyser::new (portable.rs:189-229) */
int or_analyser_portable(const or_super_opts *sopts, int32_t bw, int32_t bh, int32_t overlap_mode,
                         int32_t vectors, or_analyse_opts *out, char *err, size_t err_len);
void or_output_block(const or_analyse_opts *o, int32_t *bw, int32_t *bh, int32_t *ox, int32_t *oy);
void or_grid(const or_analyse_opts *o, int32_t bw, int32_t bh, int32_t ox, int32_t oy,
             int32_t *gw, int32_t *gh);
void or_level_grid(const or_analyse_opts *o, int32_t level, int32_t *gw, int32_t *gh);

/* ---- Super (super_build.rs) ---- */
void or_build_plane(or_px *dst, size_t dst_len, size_t dst_stride, const or_px *src,
                    size_t src_len, size_t src_stride, size_t src_w, size_t src_h, size_t luma_w,
                    size_t luma_h, int32_t chroma, const or_super_opts *o);
/* SuperBuilder::build (portable.rs:94-148): src = packed I420 (w*h + 2*(w/2*h/2)),
 * out = y (w*H) | u (w/2*H/2) | v (w/2*H/2), H = super height. */
void or_build_super_portable(const or_super_opts *o, const or_px *src, or_px *out);
size_t or_super_output_len(const or_super_opts *o);

/* ---- Analyse (analyse_search.rs) ---- */
/* analyse_pair: bwd/fwd are gw*gh arrays of the OUTPUT grid (or NULL when that
 * direction is not requested). Returns 0 or -1 when the level-0 grid is smaller than
 * 2x2 (the reference indexes field[-1] there and panics, analyse_search.rs:534-535). */
int or_analyse_pair(const or_planes *cur, const or_planes *ref, const or_analyse_opts *o,
                    or_vec8 *bwd, or_vec8 *fwd);
size_t or_payload_len(const or_analyse_opts *o);
void or_pack_vector_frame(const or_analyse_opts *o, const or_vec8 *previous, const or_vec8 *current,
                          uint8_t *out);
void or_pack_vdata_header(const or_analyse_opts *o, int32_t out[16]);
/* Analyser::analyse over two portable super frames -> payload bytes. */
int or_analyse_portable(const or_analyse_opts *o, const or_super_opts *so, const or_px *cur_super,
                        const or_px *ref_super, uint8_t *payload);
/* Clip driver used by the CPU baseline: frame n pairs with min(n+delta, nframes-1)
 * (analyse_filter.rs:277-279); pairs [first, first+count) are analysed on `threads`
 * host threads (frames in parallel, fwd/bwd as two tasks, analyse_search.rs:160-191).
 * supers[i] points at the portable super frame of frame i. */
int or_analyse_clip(const or_analyse_opts *o, const or_super_opts *so, const or_px *const *supers,
                    int32_t nframes, int32_t first, int32_t count, uint8_t *payloads, int32_t threads);
/* Super over many frames on `threads` host threads. */
void or_build_super_many(const or_super_opts *o, const or_px *const *src, or_px *const *out,
                         int32_t nframes, int32_t threads);

/* ---- consumers of the payload (svpflow-core metadata.rs / renderer.rs) ---- */
void or_vector_grid(const int32_t vdata[16], int32_t *mw, int32_t *mh);
/* decode_vectors + vector_planes for both sets; out = mvx0 | mvy0 | mvx1 | mvy1 (mw x mh each);
 * returns -1 when the payload does not decode (the reference's None). */
/* ---- SmoothFps single-warp render (renderer.rs render_mode1_or_2 without masks), 8-bit ---- */
typedef struct {
    int32_t width, height, block_w, block_h, origin_x, origin_y, grid_w, grid_h, chroma_y_div, source_step;
} or_render_config;
/* A source plane: linear (shift 0) or a super clip's level 0 with its 2^shift x 2^shift sub-planes
 * `span` bytes apart (renderer.rs Plane::super_plane). */
typedef struct {
    const uint8_t *data;
    size_t len, stride, span;
    uint32_t shift;
} or_rplane;
void or_render_luts(int32_t threshold, int16_t inverse_lut[2048], int16_t threshold_lut[2048]);
/* mask: NULL, or the mode's mask plane (grid_w x grid_h bytes, renderer.rs MaskPlanes): each sample
 * becomes mode1_pixel(base, warped, alpha) */
void or_render_warp_plane(const or_render_config *c, int32_t chroma, int32_t interp, const int16_t *lut,
                          const or_rplane *src, const uint16_t *mx, const uint16_t *my, size_t mlen,
                          const uint8_t *mask, uint8_t *dst, size_t dst_stride, size_t dst_len);
/* render_mode11_or_13 (renderer.rs:330-438) / render_mode21_or_22 (:571-641) for one plane, mode 11,
 * 13, 21 or 22; zero_origin: the interpolation grid starts at 0 (the zero-origin variant, or
 * !interp); masks a, b (both or neither for 11 / 13, both for 21 / 22) and the final mask (21 / 22,
 * optional, blending towards blend_256(cur0, cur1, threshold_limit)). */
void or_render_dual_plane(const or_render_config *c, int32_t chroma, int32_t interp, int32_t zero_origin,
                          int32_t mode, int32_t threshold, int32_t threshold_limit, const or_rplane *src0,
                          const or_rplane *src1, const uint16_t *mx0, const uint16_t *my0, const uint16_t *mx1,
                          const uint16_t *my1, size_t mlen, const uint8_t *mask_a, const uint8_t *mask_b,
                          const uint8_t *mask_f, uint8_t *dst, size_t dst_stride, size_t dst_len);
/* render_mode23 (renderer.rs:644-666) for one plane: motion sets base0, base1, next0, prev1 (mxs / mys),
 * masks a, b (required) and the optional final mask. */
void or_render_mode23_plane(const or_render_config *c, int32_t chroma, int32_t interp, int32_t threshold,
                            const or_rplane *src0, const or_rplane *src1, const uint16_t *const mxs[4],
                            const uint16_t *const mys[4], size_t mlen, const uint8_t *mask_a, const uint8_t *mask_b,
                            const uint8_t *mask_f, uint8_t *dst, size_t dst_stride, size_t dst_len);
/* set_threshold_value (renderer.rs:256-264): threshold_limit for a mask scale */
int32_t or_render_threshold_limit(int32_t threshold, double scale);
int or_vector_planes(const int32_t vdata[16], const uint8_t *payload, size_t len, int32_t frame_w, int32_t frame_h,
                     int32_t raw, uint16_t *out);
/* SmoothFps' mask planes for one payload at `phase` (0..256): out = cover0 | cover1 | area0 | area1 |
 * max(area0, area1), mw x mh bytes each (coverage_mask at 256 - phase / phase with `cover` percent,
 * magnitude_mask with area_scale, area_sharp); -1 when the payload does not decode. */
int or_render_masks(const int32_t vdata[16], const uint8_t *payload, size_t len, int32_t phase, int32_t cover,
                    double area_scale, double area_sharp, uint8_t *out);
/* SmoothFps's scene class (0..3) of one payload with the scene.luma gamma and the scene limits;
 * -1 when the payload does not decode. */
int32_t or_scene_class(const int32_t vdata[16], const uint8_t *payload, size_t len, double gamma, int32_t blocks_pct,
                       int32_t zero, int32_t m1, int32_t m2, int32_t scene);

/* ---- primitives exposed for known-answer tests ---- */
uint32_t or_hadamard4_satd(const int32_t diff[16]);
int32_t or_adapt_lambda(int32_t nlambda, int32_t lsad, uint32_t pred_score);
int32_t or_exact_lambda(const or_analyse_opts *o, int32_t level, int32_t pel);
void or_rescale_scores(or_vec8 *field, size_t n, int32_t width, int32_t height, int32_t blk);
void or_global_doubled(const or_vec8 *field, size_t n, int32_t *gx, int32_t *gy);
/* Cost of one candidate: (luma, chroma) exactly as block_cost_lc (analyse_search.rs:1683). */
void or_block_cost_lc(const or_planes *src, const or_planes *ref, int32_t level, int32_t px,
                      int32_t py, int32_t bw, int32_t bh, int32_t mvx, int32_t mvy, int32_t satd,
                      int32_t pel, uint32_t *luma, uint32_t *chroma);
/* Work counters of the last or_analyse_pair on this thread (cost evaluations,
 * luma and chroma pixels compared): the algorithmic work of the control flow. */
/* instrumentation: [0] cost evaluations, [1] / [2] luma / chroma samples compared, [3] / [4] of
 * those under SATD; for the calling thread's last pair, or summed over all pairs since the last
 * reset (or_total_counters). */
void or_last_counters(uint64_t out[5]);
void or_total_counters(uint64_t out[5], int32_t reset);
void or_level_counters(uint64_t out[64]);

#ifdef __cplusplus
}
#endif
#endif
