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

cudaError_t launch_analyse(const AnalyseParams &P, const PairSrc &src, int npairs, uint8_t *payloads,
                           uint8_t *scratch, int *status_dev, cudaStream_t stream, int *launches) {
    return nt128::launch_plain(P, src, npairs, payloads, scratch, status_dev, stream, launches);
}

}  // namespace svpf
