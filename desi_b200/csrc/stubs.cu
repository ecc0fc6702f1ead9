// stubs.cu -- entry points of include/pcf.h whose kernels are not in this
// build yet; they report PCF_ERR_UNSUPPORTED instead of computing anything.
#include "pcf_internal.cuh"

extern "C" {
}
