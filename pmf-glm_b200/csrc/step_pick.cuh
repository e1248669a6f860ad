// Lookup of the step-kernel instantiations for one tile height (included by step_ty*.cu).
#pragma once
#include "dispatch.h"
#include "step_kernel.cuh"

namespace pmf {
namespace detail {
template <int TY, int RECON, int RSOL>
StepKernel pick(bool ct, bool comp, int src) {
  if (src == SRC_DRAG)
    return ct ? mhd_step_kernel<TY, RECON, RSOL, true, false, SRC_DRAG> : mhd_step_kernel<TY, RECON, RSOL, false, false, SRC_DRAG>;
  if (src == SRC_RAD)
    return ct ? mhd_step_kernel<TY, RECON, RSOL, true, false, SRC_RAD> : mhd_step_kernel<TY, RECON, RSOL, false, false, SRC_RAD>;
  if (ct)
    return comp ? mhd_step_kernel<TY, RECON, RSOL, true, true, SRC_NONE>
                : mhd_step_kernel<TY, RECON, RSOL, true, false, SRC_NONE>;
  return comp ? mhd_step_kernel<TY, RECON, RSOL, false, true, SRC_NONE>
              : mhd_step_kernel<TY, RECON, RSOL, false, false, SRC_NONE>;
}
template <int TY, int RECON, int RSOL>
BatchKernel pick_batch(bool ct, bool comp) {
  if (ct) return comp ? mhd_batch_kernel<TY, RECON, RSOL, true, true> : mhd_batch_kernel<TY, RECON, RSOL, true, false>;
  return comp ? mhd_batch_kernel<TY, RECON, RSOL, false, true> : mhd_batch_kernel<TY, RECON, RSOL, false, false>;
}
template <int TY, int RECON>
BatchKernel pick_batch_rs(int rsol, bool ct, bool comp) {
  switch (rsol) {
    case RS_HLLD: return pick_batch<TY, RECON, RS_HLLD>(ct, comp);
    case RS_HLL: return pick_batch<TY, RECON, RS_HLL>(ct, comp);
    case RS_LLF: return pick_batch<TY, RECON, RS_LLF>(ct, comp);
  }
  return nullptr;
}
template <int TY>
BatchKernel batch(int recon, int rsol, bool ct, bool comp) {
  switch (recon) {
    case RECON_PLM: return pick_batch_rs<TY, RECON_PLM>(rsol, ct, comp);
    case RECON_PPM: return pick_batch_rs<TY, RECON_PPM>(rsol, ct, comp);
    case RECON_PLM_MINMOD: return pick_batch_rs<TY, RECON_PLM_MINMOD>(rsol, ct, comp);
  }
  return nullptr;
}
template <int TY, int RECON>
StepKernel pick_rs(int rsol, bool ct, bool comp, int src) {
  switch (rsol) {
    case RS_HLLD: return pick<TY, RECON, RS_HLLD>(ct, comp, src);
    case RS_HLL: return pick<TY, RECON, RS_HLL>(ct, comp, src);
    case RS_LLF: return pick<TY, RECON, RS_LLF>(ct, comp, src);
  }
  return nullptr;
}
template <int TY>
StepKernelInfo info(int recon, int rsol, bool ct, bool comp, int src) {
  StepKernelInfo k{nullptr, StepSmem<TY>::BYTES, step_threads<TY>()};
  switch (recon) {
    case RECON_PLM: k.fn = pick_rs<TY, RECON_PLM>(rsol, ct, comp, src); break;
    case RECON_PPM: k.fn = pick_rs<TY, RECON_PPM>(rsol, ct, comp, src); break;
    case RECON_PLM_MINMOD: k.fn = pick_rs<TY, RECON_PLM_MINMOD>(rsol, ct, comp, src); break;
  }
  return k;
}
}  // namespace detail
}  // namespace pmf
