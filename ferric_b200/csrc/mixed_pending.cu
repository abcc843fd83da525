// Split-BF16 entry points that are not built yet report FC_ERR_KERNEL
// (never a silent FP64 run).
#include "fc_internal.cuh"
#include "rimp2.cuh"
#include "dfjk.cuh"

namespace fc {
fc_status dfjk_prepare_mixed(fc_dfjk*, cudaStream_t) {
    return fail(FC_ERR_KERNEL, "split-BF16 DF-JK kernels not available in this build");
}
void dfjk_free_mixed(fc_dfjk*) {}
fc_status dfj_build_mixed(fc_dfjk*, const double*, double*, cudaStream_t, fc_stats*) {
    return fail(FC_ERR_KERNEL, "split-BF16 DF-J kernel not available in this build");
}
fc_status dfk_build_mixed(fc_dfjk*, const double*, int64_t, double*, cudaStream_t, fc_stats*) {
    return fail(FC_ERR_KERNEL, "split-BF16 DF-K kernel not available in this build");
}
}  // namespace fc
