// Host-side dispatch over the instantiated tile heights.
#include "dispatch.h"

namespace pmf {
StepKernelInfo step_kernel_info_ty5(int recon, int rsol, bool ct, bool comp, int src);
StepKernelInfo step_kernel_info_ty8(int recon, int rsol, bool ct, bool comp, int src);
StepKernelInfo step_kernel_info_ty9(int recon, int rsol, bool ct, bool comp, int src);
StepKernelInfo step_kernel_info_ty13(int recon, int rsol, bool ct, bool comp, int src);

BatchKernel batch_kernel_ty5(int recon, int rsol, bool ct, bool comp);
BatchKernel batch_kernel_ty8(int recon, int rsol, bool ct, bool comp);
BatchKernel batch_kernel_ty9(int recon, int rsol, bool ct, bool comp);
BatchKernel batch_kernel_ty13(int recon, int rsol, bool ct, bool comp);

BatchKernel batch_kernel(int ty, int recon, int rsol, bool ct, bool comp) {
  switch (ty) {
    case 5: return batch_kernel_ty5(recon, rsol, ct, comp);
    case 8: return batch_kernel_ty8(recon, rsol, ct, comp);
    case 9: return batch_kernel_ty9(recon, rsol, ct, comp);
    case 13: return batch_kernel_ty13(recon, rsol, ct, comp);
  }
  return nullptr;
}

StepKernelInfo step_kernel_info(int ty, int recon, int rsol, bool ct, bool comp, int src) {
  switch (ty) {
    case 5: return step_kernel_info_ty5(recon, rsol, ct, comp, src);
    case 8: return step_kernel_info_ty8(recon, rsol, ct, comp, src);
    case 9: return step_kernel_info_ty9(recon, rsol, ct, comp, src);
    case 13: return step_kernel_info_ty13(recon, rsol, ct, comp, src);
  }
  return StepKernelInfo{nullptr, 0, 0};
}
}  // namespace pmf
