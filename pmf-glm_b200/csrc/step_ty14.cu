// Step-kernel instantiations for CTAs of 14 owned rows.
#include "step_pick.cuh"

namespace pmf {
StepKernelInfo step_kernel_info_ty14(int recon, int rsol, bool ct, bool comp) {
  return detail::info<14>(recon, rsol, ct, comp);
}
BatchKernel batch_kernel_ty14(int recon, int rsol, bool ct, bool comp) {
  return detail::batch<14>(recon, rsol, ct, comp);
}
}  // namespace pmf
