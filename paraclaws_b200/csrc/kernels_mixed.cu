// kernels_mixed.cu -- mixed-precision precision form (FP32 flux/limiter, FP64 state).
#include "../../include/paraclaws_b200.h"
#include "pcl_mixed.h"

namespace pcl {
int mixed_create(const GridDev&, cudaStream_t, void** ws) {
  *ws = nullptr;
  return PCL_ERR_BADARG;
}
void mixed_free(void*) {}
void launch_sweeps_mixed(const GridDev&, void*, cudaStream_t) {}
}  // namespace pcl
