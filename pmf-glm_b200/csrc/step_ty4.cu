// Step-kernel instantiations for CTAs of 4 owned rows.
#include "step_pick.cuh"

namespace pmf {
StepKernelInfo step_kernel_info_ty4(int recon, int rsol, bool ct, bool comp) {
  return detail::info<4>(recon, rsol, ct, comp);
}
BatchKernel batch_kernel_ty4(int recon, int rsol, bool ct, bool comp) {
  return detail::batch<4>(recon, rsol, ct, comp);
}
}  // namespace pmf
