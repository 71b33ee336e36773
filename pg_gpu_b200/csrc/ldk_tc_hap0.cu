// Haplotype path, default tile.
#include "ldk_tc_kernel.cuh"

namespace ldk {
cudaError_t launch_tc_hap_v0(const ldk_parse_t* d, const ldk_parse_out_t* o, const Scratch& w, const ParseShape& sh,
                             int max_items, cudaStream_t s) {
    return dispatch_tc<false, 0, double>(d, o, w, sh, max_items, s);
}
}  // namespace ldk
