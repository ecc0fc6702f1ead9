// stubs.cu -- entry points of include/pcf.h whose kernels are not in this
// build yet; they report PCF_ERR_UNSUPPORTED instead of computing anything.
#include "pcf_internal.cuh"

extern "C" {
}

pcf_status pcf_count_triplets_ani(pcf_ctx *, const pcf_grid *, const pcf_grid *, int, float,
                                  uint32_t, double *, pcf_stats *) {
    return PCF_ERR_UNSUPPORTED;
}
