// The HLLD degeneracy census step: the fused GLM step (8 owned rows, MC-PLM, plain update)
// with HLLD counting its single-star degeneracy cases (RS_HLLD_CENSUS).
#include "dispatch.h"
#include "step_kernel.cuh"

namespace pmf {
StepKernelInfo step_census_kernel_info() {
  return StepKernelInfo{mhd_step_kernel<kCensusRows, RECON_PLM, RS_HLLD_CENSUS, false, false, SRC_NONE>,
                        StepSmem<kCensusRows>::BYTES, step_threads<kCensusRows>()};
}
}  // namespace pmf
