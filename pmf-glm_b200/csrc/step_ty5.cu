// Step-kernel instantiations for CTAs of 5 owned rows.
#include "step_pick.cuh"

namespace pmf {
StepKernelInfo step_kernel_info_ty5(int recon, int rsol, bool ct, bool comp, int src) {
  return detail::info<5>(recon, rsol, ct, comp, src);
}
BatchKernel batch_kernel_ty5(int recon, int rsol, bool ct, bool comp) {
  return detail::batch<5>(recon, rsol, ct, comp);
}
}  // namespace pmf
