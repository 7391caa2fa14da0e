// variants.cpp -- the table of compiled Analyse launch shapes (one TU per shape).
#include "svpf_device.h"

namespace svpf {

namespace {
const AnalyseVariant kVariants[] = {
    {"nt128_b2", 128, 2, nt128::launch_plain, nt128::batch_blocks_per_sm, nt128::launch_batch},
    {"nt64_b4", 64, 4, nt64::launch_plain, nt64::batch_blocks_per_sm, nt64::launch_batch},
    {"nt32_b8", 32, 8, nt32::launch_plain, nt32::batch_blocks_per_sm, nt32::launch_batch},
    {"nt128_b3", 128, 3, nt128b3::launch_plain, nt128b3::batch_blocks_per_sm, nt128b3::launch_batch},
    {"nt64_b6", 64, 6, nt64b6::launch_plain, nt64b6::batch_blocks_per_sm, nt64b6::launch_batch},

};
}  // namespace

int analyse_variant_count() { return (int)(sizeof(kVariants) / sizeof(kVariants[0])); }
const AnalyseVariant &analyse_variant(int i) {
    return kVariants[(i >= 0 && i < analyse_variant_count()) ? i : 0];
}

// The 128-register shape, whose level 0 spreads over the GPU by default; with that off, more
// pairs than two per SM take the 80-register shape (three pairs per SM resident). uint16
// samples have one compiled shape.
cudaError_t launch_analyse(const AnalyseParams &P, const PairSrc &src, int npairs, uint8_t *payloads,
                           uint8_t *scratch, int *status_dev, cudaStream_t stream, int *launches) {
    if (P.px_bytes == 2) return nt128p16::launch_plain(P, src, npairs, payloads, scratch, status_dev, stream, launches);
    static int sms = [] {
        int dev = 0, n = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            return 0;
        return n;
    }();
    // more pairs than two per SM: the 3-CTA shape, unless level 0 is spread over the GPU, which
    // balances the SMs at any pair count (900 pairs at 960x540: 581.9 -> 754.1 pairs/s)
    if (sms > 0 && npairs > 2 * sms && (P.lookahead & 5) != 5)
        return nt128b3::launch_plain(P, src, npairs, payloads, scratch, status_dev, stream, launches);
    return nt128::launch_plain(P, src, npairs, payloads, scratch, status_dev, stream, launches);
}

cudaError_t launch_analyse_shape(int variant, const AnalyseParams &P, const PairSrc &src, int npairs, uint8_t *payloads,
                                 uint8_t *scratch, int *status_dev, cudaStream_t stream, int *launches) {
    if (P.px_bytes == 2) return nt128p16::launch_plain(P, src, npairs, payloads, scratch, status_dev, stream, launches);
    return analyse_variant(variant).launch_plain(P, src, npairs, payloads, scratch, status_dev, stream, launches);
}

}  // namespace svpf
