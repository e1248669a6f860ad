// Lookup of the step-kernel instantiations for one tile height (included by step_ty*.cu).
#pragma once
#include "dispatch.h"
#include "step_kernel.cuh"

namespace pmf {
namespace detail {
template <int TY, int RECON, int RSOL>
StepKernel pick(bool ct, bool comp, bool drag) {
  if (drag) return ct ? mhd_step_kernel<TY, RECON, RSOL, true, false, true> : mhd_step_kernel<TY, RECON, RSOL, false, false, true>;
  if (ct)
    return comp ? mhd_step_kernel<TY, RECON, RSOL, true, true, false> : mhd_step_kernel<TY, RECON, RSOL, true, false, false>;
  return comp ? mhd_step_kernel<TY, RECON, RSOL, false, true, false> : mhd_step_kernel<TY, RECON, RSOL, false, false, false>;
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
StepKernel pick_rs(int rsol, bool ct, bool comp, bool drag) {
  switch (rsol) {
    case RS_HLLD: return pick<TY, RECON, RS_HLLD>(ct, comp, drag);
    case RS_HLL: return pick<TY, RECON, RS_HLL>(ct, comp, drag);
    case RS_LLF: return pick<TY, RECON, RS_LLF>(ct, comp, drag);
  }
  return nullptr;
}
template <int TY>
StepKernelInfo info(int recon, int rsol, bool ct, bool comp, bool drag) {
  StepKernelInfo k{nullptr, StepSmem<TY>::BYTES, step_threads<TY>()};
  switch (recon) {
    case RECON_PLM: k.fn = pick_rs<TY, RECON_PLM>(rsol, ct, comp, drag); break;
    case RECON_PPM: k.fn = pick_rs<TY, RECON_PPM>(rsol, ct, comp, drag); break;
    case RECON_PLM_MINMOD: k.fn = pick_rs<TY, RECON_PLM_MINMOD>(rsol, ct, comp, drag); break;
  }
  return k;
}
}  // namespace detail
}  // namespace pmf
