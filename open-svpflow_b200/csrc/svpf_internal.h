// svpf_internal.h -- internal types of the B200 motion-analysis library (host + device).
//
// Option structs mirror crates/svpflow1/src/super_opts.rs:3-14 (SuperOpts) and
// crates/svpflow1/src/analyse_opts.rs:4-42 (AnalyseOpts); the device parameter block
// (AnalyseParams) is this library's own precomputation of every per-level scalar the
// search needs, so the kernel reads them from the parameter space instead of recomputing.
#pragma once
#include <stddef.h>
#include <stdint.h>

#include <string>

namespace svpf {

constexpr int kMaxLevels = 16;

struct SuperOpts {
    int32_t pel = 2, gpu = 1, scale_down = 4, scale_up = 0;
    int32_t full = 1, rc = 0;
    int32_t levels = 0, width = 0, height = 0;
    int32_t bits = 8;  // sample depth: 8 (the reference) or 10 (this project's extension, uint16 samples)
};

struct AnalyseOpts {
    int32_t vectors, block_w, block_h, overlap_mode, overlap_x, overlap_y, delta, pel, selector;
    int32_t levels, super_levels, width, height, lambda, lsad;
    double plevel;
    int32_t pnew, pglobal, pzero, pnbour, prev;
    int32_t search_type, coarse_search_type, distance, coarse_distance;
    int32_t coarse_trymany, coarse_bad_sad, coarse_bad_range;
    int32_t fine_satd, coarse_satd;
    int32_t has_refine_thsad, refine_thsad, refine_search_type, refine_distance, refine_satd;
    int32_t sort;
};

// Byte layout of one super frame in memory: Y plane (y_stride x super_h rows), then
// U and V planes (c_stride x super_h/2 rows each). The portable layout of
// crates/svpflow1/src/portable.rs:104-106 is y_stride = width, c_stride = width/2.
struct SuperLayout {
    int32_t width, height, pel, levels, full, super_h;
    int64_t y_stride, c_stride;         // in samples
    int64_t y_len, c_len;               // plane sizes in samples
    int64_t frame_bytes;                // (y + u + v) * px_bytes
    int32_t px_bytes;                   // 1 (8-bit) or 2 (uint16 samples)
};

// ---- options (opts.cpp) ----
// Parsed opt-string tree of crates/svpflow-core/src/params.rs (lenient JSON).
struct OptValue;
struct OptTree {
    OptValue *root = nullptr;
    OptTree() = default;
    OptTree(const OptTree &) = delete;
    OptTree &operator=(const OptTree &) = delete;
    ~OptTree();
};
// Returns false (and fills err) on a syntax error, like params::parse.
bool parse_opt(const char *text, size_t len, OptTree &out, std::string &err);

int32_t reduce_dim(int32_t dim, int32_t n);
int32_t auto_levels(int32_t width, int32_t height);
int32_t super_plane_height(int32_t base_h, int32_t pel, int32_t levels, bool full);
bool super_opts_from_opt(const OptTree *opt, int32_t width, int32_t height, SuperOpts &o, std::string &err);
int64_t super_pack_data(const SuperOpts &o);
bool analyse_opts_from_opt(const OptTree *opt, int64_t sdata, const SuperOpts *hint, AnalyseOpts &o,
                           std::string &err);
bool analyse_opts_portable(const SuperOpts &so, int32_t bw, int32_t bh, int32_t overlap_mode, int32_t vectors,
                           AnalyseOpts &o, std::string &err);
bool overlap_from_mode(int32_t bw, int32_t bh, int32_t mode, int32_t &ox, int32_t &oy, std::string &err);
int32_t auto_search_levels(int32_t w, int32_t h, int32_t bw, int32_t bh, int32_t ox, int32_t oy);
void output_block(const AnalyseOpts &o, int32_t &bw, int32_t &bh, int32_t &ox, int32_t &oy);
void output_grid(const AnalyseOpts &o, int32_t bw, int32_t bh, int32_t ox, int32_t oy, int32_t &gw, int32_t &gh);
void level_grid(const AnalyseOpts &o, int32_t level, int32_t &gw, int32_t &gh);
size_t payload_len(const AnalyseOpts &o);
void vdata_header(const AnalyseOpts &o, int32_t h[16]);
SuperLayout portable_layout(const SuperOpts &so);
// The same planes with other row pitches (a frame server's frames): Y y_stride x H, then U
// and V c_stride x H/2 each, contiguous.
SuperLayout strided_layout(const SuperOpts &so, int64_t y_stride, int64_t c_stride);

// ---- device parameter block for one Analyse configuration (analyse.cu) ----
struct LevelInfo {
    int32_t gw, gh;           // level grid incl. the extra edge row/column at level > 0
    int32_t lw, lh;           // reduce_dim(luma_w/h, level)
    int64_t y_off, c_off;     // first row of the level in the Y / chroma planes
    int32_t pel;              // opts.pel at level 0, else 1
    int32_t lambda_base;      // exact_lambda (0 at the smallest level)
    int32_t lsad;             // opts.lsad, /3 at the smallest level
    int32_t satd, search_type, base_radius, smallest;
    int32_t bw, bh, pxoff, pyoff;  // searched block (halved and centred at the smallest level)
    int32_t tl, tc;           // 4x4 luma tiles, 4x4 chroma tiles per plane of one candidate
};

struct alignas(16) AnalyseParams {
    int32_t nlevels;
    LevelInfo lv[kMaxLevels];
    int32_t block_w, block_h, ox, oy, step_x, step_y;
    int32_t pnew, prev, pzero, pglobal, pnbour, distance;
    int32_t coarse_bad_sad, coarse_bad_range, coarse_distance, vectors;
    int32_t luma_w, luma_h, pel;
    int64_t y_stride, c_stride, y_len, c_len, frame_bytes;
    // output grid (after the optional refine pass)
    int32_t out_gw, out_gh, out_bw, out_bh, out_ox, out_oy;
    int32_t has_refine, refine_thsad, refine_search_type, refine_distance, refine_satd, lambda;
    LevelInfo rlv[2];         // refine pass block shapes: output block, half of it (border blocks)
    int32_t rescale_denom;
    int32_t tiles_per_lane;   // 4x4 tiles one lane evaluates per candidate (2, 4 or 8): a launch tuning knob
    int32_t px_bytes;         // 1: 8-bit samples; 2: uint16 samples (the 10-bit extension)
    int32_t lookahead;        // look-ahead (one block per warp in flight, exact either way): bit 0 level 0,
                              // bit 1 the coarser levels (slower: measured), bit 2 level 0 spread over
                              // the GPU (its own launch, one CTA per warp); a tuning knob, default 5
    int32_t pad0_, pad1_, pad2_;
    int64_t payload_len;
    int32_t header[16];       // payload words 0x00..0x3C
    // per-pair scratch layout (bytes)
    int64_t max_cells, max_order;
    int64_t off_field[2], off_next[2], off_proj[2][2], off_order[2], off_order2[2], off_pos[2];
    int64_t off_keys[2], off_hist[2], off_seen[2], off_out[2];
    int64_t off_ctl[2];       // per direction: the hand-over words of the level-0 kernel (CTL_*)
    int64_t scratch_per_pair;
};

static_assert(sizeof(AnalyseParams) % 16 == 0, "AnalyseParams is copied in 16-byte words");

bool build_analyse_params(const AnalyseOpts &o, const SuperLayout &L, AnalyseParams &P, std::string &err);

}  // namespace svpf
