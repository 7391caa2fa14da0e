// params.cpp -- host-side precomputation of the device parameter block of one Analyse
// configuration: per-level grids, plane offsets, lambdas, radii, the payload header and
// the per-pair scratch layout. Follows crates/svpflow1/src/analyse_search.rs (level
// offsets :49-58 and :2704-2713, exact_lambda :1279-1283, search_radius :1465-1476,
// rescale_scores :2716-2721, pack_vector_frame :2740-2811).
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <string>

#include "svpf_internal.h"

namespace svpf {

bool build_analyse_params(const AnalyseOpts &o, const SuperLayout &Lay, AnalyseParams &P, std::string &err) {
    memset(&P, 0, sizeof(P));
    if (o.levels < 1 || o.levels > kMaxLevels) { err = "unsupported level count"; return false; }
    if (!Lay.full) { err = "SVAnalyse: the super clip must hold the finest level (full=true)"; return false; }
    P.nlevels = o.levels;
    P.block_w = o.block_w; P.block_h = o.block_h; P.ox = o.overlap_x; P.oy = o.overlap_y;
    P.step_x = o.block_w - o.overlap_x > 1 ? o.block_w - o.overlap_x : 1;
    P.step_y = o.block_h - o.overlap_y > 1 ? o.block_h - o.overlap_y : 1;
    P.pnew = o.pnew; P.prev = o.prev; P.pzero = o.pzero; P.pglobal = o.pglobal; P.pnbour = o.pnbour;
    P.distance = o.distance; P.coarse_bad_sad = o.coarse_bad_sad; P.coarse_bad_range = o.coarse_bad_range;
    P.coarse_distance = o.coarse_distance; P.vectors = o.vectors;
    P.luma_w = o.width; P.luma_h = o.height; P.pel = o.pel;
    if (Lay.y_len >= (int64_t)1 << 30 || Lay.c_len >= (int64_t)1 << 30) {  // offsets are 32-bit on the device
        err = "SVAnalyse: super frames of 2^30 bytes or more are not available on the device path";
        return false;
    }
    P.y_stride = Lay.y_stride; P.c_stride = Lay.c_stride; P.y_len = Lay.y_len; P.c_len = Lay.c_len;
    P.frame_bytes = Lay.frame_bytes;
    P.px_bytes = Lay.px_bytes;
    P.lambda = o.lambda;
    P.tiles_per_lane = 8;
    P.lookahead = 5;
    // per level
    int64_t max_cells = 1, max_order = 1;
    for (int lv = 0; lv < o.levels; lv++) {
        LevelInfo &L = P.lv[lv];
        level_grid(o, lv, L.gw, L.gh);
        L.lw = reduce_dim(o.width, lv);
        L.lh = reduce_dim(o.height, lv);
        int64_t y = 0, c = 0;  // level_y_offset / chroma_level_offset (:49-58, :2704-2713)
        for (int k = 0; k < lv; k++) {
            const int64_t h = reduce_dim(Lay.height, k);
            const int64_t sub = (k == 0 && Lay.full) ? (int64_t)Lay.pel * Lay.pel : 1;
            y += h * sub;
            const int64_t hc = h / 2;
            c += (hc > 1 ? hc : 1) * sub;
        }
        L.y_off = y; L.c_off = c;
        L.pel = lv == 0 ? (o.pel > 1 ? o.pel : 1) : 1;
        L.smallest = lv == o.levels - 1;
        // exact_lambda (:1279-1283), f64: lambda / plevel^(levels-level-1) / pel^2
        {
            double a = o.plevel, r = 1.0;
            int b = o.levels - lv - 1;
            for (;;) {  // compiler-rt __powidf2 order
                if (b & 1) r *= a;
                b /= 2;
                if (b == 0) break;
                a *= a;
            }
            const double v = (double)o.lambda / r / (double)((L.pel * L.pel) > 1 ? L.pel * L.pel : 1);
            int32_t iv;
            if (v != v) iv = 0;
            else if (v >= 2147483647.0) iv = INT32_MAX;
            else if (v <= -2147483648.0) iv = INT32_MIN;
            else iv = (int32_t)v;
            L.lambda_base = L.smallest ? 0 : iv;
        }
        L.lsad = L.smallest ? o.lsad / 3 : o.lsad;
        L.satd = lv == 0 ? o.fine_satd : o.coarse_satd;
        L.search_type = lv == 0 ? o.search_type : o.coarse_search_type;
        {  // search_radius (:1465-1476)
            const int dd = lv == 0 ? o.distance : o.coarse_distance;
            const int nl = o.levels > 1 ? o.levels : 1;
            L.base_radius = dd == 0 ? ((lv == 0 && nl > 1) ? 0 : 10) : (dd < 0 ? -dd : dd);
        }
        if (L.smallest) {
            L.bw = o.block_w >> 1; L.bh = o.block_h >> 1; L.pxoff = o.block_w >> 2; L.pyoff = o.block_h >> 2;
        } else {
            L.bw = o.block_w; L.bh = o.block_h; L.pxoff = 0; L.pyoff = 0;
        }
        L.tl = ((L.bw + 3) / 4) * ((L.bh + 3) / 4);
        const int cw = L.bw / 2, ch = L.bh / 2;
        L.tc = cw > 0 ? ((cw + 3) / 4) * (((cw > ch ? cw : ch) + 3) / 4) : 0;
        const int64_t cells = (int64_t)L.gw * L.gh;
        if (cells > max_cells) max_cells = cells;
        const int64_t ol = cells + L.gw + L.gh + 8;
        if (ol > max_order) max_order = ol;
        if (L.tl + L.tc > 96 || L.gw > 65535 || L.gh > 65535) { err = "unsupported block / grid size"; return false; }
    }
    {  // level-0 grid must be at least 2x2: below that the reference indexes field[-1]
        if (P.lv[0].gw < 2 || P.lv[0].gh < 2) { err = "SVAnalyse: frame too small for the block grid"; return false; }
    }
    int32_t bw, bh, ox, oy, gw, gh;
    output_block(o, bw, bh, ox, oy);
    output_grid(o, bw, bh, ox, oy, gw, gh);
    P.out_bw = bw; P.out_bh = bh; P.out_ox = ox; P.out_oy = oy; P.out_gw = gw; P.out_gh = gh;
    P.has_refine = o.has_refine_thsad;
    P.refine_thsad = o.refine_thsad;
    P.refine_search_type = o.refine_search_type;
    P.refine_distance = o.refine_distance;
    P.refine_satd = o.refine_satd;
    if (P.has_refine) {  // exact_recalculate (:1326-1451) block shapes at level 0
        for (int k = 0; k < 2; k++) {
            LevelInfo &R = P.rlv[k];
            R = P.lv[0];
            R.gw = gw; R.gh = gh;
            R.bw = k ? bw / 2 : bw; R.bh = k ? bh / 2 : bh;
            R.pxoff = 0; R.pyoff = 0; R.smallest = 0; R.lambda_base = 0; R.lsad = 0;
            R.satd = o.refine_satd;
            R.search_type = o.refine_search_type;
            R.base_radius = o.refine_distance < 0 ? -o.refine_distance : o.refine_distance;
            R.tl = ((R.bw + 3) / 4) * ((R.bh + 3) / 4);
            const int cw = R.bw / 2, ch = R.bh / 2;
            R.tc = cw > 0 ? ((cw + 3) / 4) * (((cw > ch ? cw : ch) + 3) / 4) : 0;
            if (R.tl + R.tc > 96) { err = "unsupported block / grid size"; return false; }
        }
        if ((int64_t)gw * gh > max_cells) max_cells = (int64_t)gw * gh;
    }
    {  // rescale_scores denominators (:2716-2721)
        double f = sqrt((double)o.width * (double)o.width + (double)o.height * (double)o.height);
        int32_t diag = f != f ? 0 : (f >= 2147483647.0 ? INT32_MAX : (int32_t)f);
        if (diag < 0) diag = 0;
        int64_t den = (int64_t)diag * (bw > 1 ? bw : 1);
        if (den > INT32_MAX) den = INT32_MAX;
        P.rescale_denom = den > 1 ? (int32_t)den : 1;
    }
    P.payload_len = (int64_t)payload_len(o);
    int32_t hdr[16];
    vdata_header(o, hdr);
    // payload words: 16, 0xA0, flags, bw, bh, pel, levels, 0, w, h, ox, oy, gw, gh, selector, delta
    P.header[0] = 16; P.header[1] = 0xA0; P.header[2] = hdr[1]; P.header[3] = bw; P.header[4] = bh;
    P.header[5] = o.pel; P.header[6] = hdr[5]; P.header[7] = 0; P.header[8] = o.width; P.header[9] = o.height;
    P.header[10] = ox; P.header[11] = oy; P.header[12] = gw; P.header[13] = gh; P.header[14] = o.selector;
    P.header[15] = o.delta;
    if (!P.has_refine && (int64_t)gw * gh != (int64_t)P.lv[0].gw * P.lv[0].gh) {
        err = "output grid differs from the level-0 grid";
        return false;
    }
    // scratch layout per pair
    int64_t np2 = 1;
    while (np2 < max_cells) np2 <<= 1;
    P.max_cells = max_cells;
    P.max_order = max_order;
    int64_t off = 0;
    auto take = [&](int64_t bytes) { int64_t o_ = off; off += (bytes + 255) & ~(int64_t)255; return o_; };
    for (int dd = 0; dd < 2; dd++) {
        P.off_field[dd] = take(max_cells * 8);
        P.off_next[dd] = take(max_cells * 8);
        P.off_proj[dd][0] = take(max_cells * 8);
        P.off_proj[dd][1] = take(max_cells * 8);
        P.off_order[dd] = take(max_order * 4);
        P.off_order2[dd] = take(max_order * 4);
        P.off_pos[dd] = take(max_cells * 4);
        P.off_keys[dd] = take(np2 * 8 > max_order * 4 ? np2 * 8 : max_order * 4);
        P.off_hist[dd] = take(65536 * 4);
        P.off_seen[dd] = take(max_cells);
        P.off_out[dd] = take(max_cells * 2);
        P.off_ctl[dd] = take(64);
    }
    P.scratch_per_pair = off;
    return true;
}

}  // namespace svpf
