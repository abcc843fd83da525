// Split-BF16 entry points that are not built yet report FC_ERR_KERNEL
// (never a silent FP64 run).
#include "fc_internal.cuh"
#include "rimp2.cuh"
#include "dfjk.cuh"

namespace fc {
fc_status dfk_build_mixed(fc_dfjk*, const double*, int64_t, double*, cudaStream_t, fc_stats*) {
    return fail(FC_ERR_KERNEL, "split-BF16 DF-K kernel not available in this build; call fc_dfjk_set_precision(h, FC_PREC_F64) for K");
}
}  // namespace fc
