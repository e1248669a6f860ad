// Instantiations of the fused step kernel and the host-side lookup table over
// (rows per CTA, reconstruction, Riemann solver, GLM/CT, plain/compensated).
#include "step_kernel.cuh"
#include "dispatch.h"

namespace pmf {

namespace {
template <int TY, int RECON, int RSOL>
StepKernel pick(bool ct, bool comp) {
  if (ct) return comp ? mhd_step_kernel<TY, RECON, RSOL, true, true> : mhd_step_kernel<TY, RECON, RSOL, true, false>;
  return comp ? mhd_step_kernel<TY, RECON, RSOL, false, true> : mhd_step_kernel<TY, RECON, RSOL, false, false>;
}
template <int TY, int RECON>
StepKernel pick_rs(int rsol, bool ct, bool comp) {
  switch (rsol) {
    case RS_HLLD: return pick<TY, RECON, RS_HLLD>(ct, comp);
    case RS_HLL: return pick<TY, RECON, RS_HLL>(ct, comp);
    case RS_LLF: return pick<TY, RECON, RS_LLF>(ct, comp);
  }
  return nullptr;
}
template <int TY>
StepKernel pick_ty(int recon, int rsol, bool ct, bool comp) {
  switch (recon) {
    case RECON_PLM: return pick_rs<TY, RECON_PLM>(rsol, ct, comp);
    case RECON_PPM: return pick_rs<TY, RECON_PPM>(rsol, ct, comp);
    case RECON_PLM_MINMOD: return pick_rs<TY, RECON_PLM_MINMOD>(rsol, ct, comp);
  }
  return nullptr;
}
}  // namespace

StepKernelInfo step_kernel_info(int ty, int recon, int rsol, bool ct, bool comp) {
  StepKernelInfo k{nullptr, 0, 0};
  switch (ty) {
    case 4:
      k.fn = pick_ty<4>(recon, rsol, ct, comp);
      k.smem_bytes = StepSmem<4>::BYTES;
      break;
    case 8:
      k.fn = pick_ty<8>(recon, rsol, ct, comp);
      k.smem_bytes = StepSmem<8>::BYTES;
      break;
    default:
      return k;
  }
  k.threads = 32 * (ty + 2);
  return k;
}

}  // namespace pmf
