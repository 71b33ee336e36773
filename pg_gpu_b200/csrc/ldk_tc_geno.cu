// Genotype path, both tiles (FP64 estimators).
#include "ldk_tc_kernel.cuh"

namespace ldk {
cudaError_t launch_tc_geno(const ldk_parse_t* d, const ldk_parse_out_t* o, const Scratch& w, const ParseShape& sh,
                           int max_items, int variant, cudaStream_t s) {
    if (variant == 1 && sh.P <= 2) return dispatch_tc<true, 1, double>(d, o, w, sh, max_items, s);
    return dispatch_tc<true, 0, double>(d, o, w, sh, max_items, s);
}
}  // namespace ldk
