// Step-kernel instantiations for CTAs of 9 owned rows.
#include "step_pick.cuh"

namespace pmf {
StepKernelInfo step_kernel_info_ty9(int recon, int rsol, bool ct, bool comp, int src) {
  return detail::info<9>(recon, rsol, ct, comp, src);
}
BatchKernel batch_kernel_ty9(int recon, int rsol, bool ct, bool comp) {
  return detail::batch<9>(recon, rsol, ct, comp);
}
}  // namespace pmf
