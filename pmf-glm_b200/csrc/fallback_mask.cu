// Fallback mask of the masked radiation step (pmfmhd_radiation_fallback_mask):
//   _radiation_fallback_mask_k!        (radiation_coupling.jl:1536-1552): the cell or one of its six
//                                      face neighbours has a negative trial density;
//   _radiation_expand_fallback_mask_k! (radiation_coupling.jl:1554-1577): the same, or the previous
//                                      mask is positive at the cell or one of its face neighbours.
// One pass over the cells with periodic neighbours (HBM-bound: 4 B read per input field and 4 B
// written per cell; the six neighbour reads come from L1/L2).
#include "aux_kernels.cuh"
#include "host_internal.h"

namespace pmf {
namespace {

template <bool EXPAND>
__global__ void __launch_bounds__(AUX_THREADS) fallback_mask_kernel(const float* __restrict__ rho,
                                                                    const float* __restrict__ prev,
                                                                    float* __restrict__ out, int nx, int ny, int nz) {
  const long long nxy = (long long)nx * ny, nc = nxy * nz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < nc; c += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(c / nxy);
    const long long r = c - (long long)k * nxy;
    const int j = (int)(r / nx), i = (int)(r - (long long)j * nx);
    // the cell and its six periodic face neighbours
    const long long nb[7] = {c,
                             c - i + (i == 0 ? nx - 1 : i - 1),
                             c - i + (i == nx - 1 ? 0 : i + 1),
                             c + ((j == 0 ? ny - 1 : j - 1) - j) * (long long)nx,
                             c + ((j == ny - 1 ? 0 : j + 1) - j) * (long long)nx,
                             c + ((k == 0 ? nz - 1 : k - 1) - k) * nxy,
                             c + ((k == nz - 1 ? 0 : k + 1) - k) * nxy};
    bool bad = false;
#pragma unroll
    for (int q = 0; q < 7; ++q) {
      bad = bad || rho[nb[q]] < 0.0f;
      if constexpr (EXPAND) bad = bad || prev[nb[q]] > 0.0f;
    }
    out[c] = bad ? 1.0f : 0.0f;
  }
}

}  // namespace
}  // namespace pmf

using namespace pmf;
using namespace pmf::host;

extern "C" {

int pmfmhd_radiation_fallback_mask(pmfmhd_ctx* c, const pmfmhd_grid* g, const float* trial_rho,
                                   const float* mask_in, float* mask_out, void* stream) {
  if (c == nullptr || trial_rho == nullptr || mask_out == nullptr) return PMFMHD_EINVAL;
  int rc = check_grid(g);
  if (rc) return rc;
  if (!all_periodic(g)) return PMFMHD_EUNSUPPORTED;
  const long long nc = ncells(g);
  // the output must not overlap an input: every cell reads its neighbours' inputs
  auto overlaps = [nc](const float* a, const float* b) { return b != nullptr && a < b + nc && b < a + nc; };
  if (overlaps(mask_out, trial_rho) || overlaps(mask_out, mask_in)) return PMFMHD_EINVAL;
  const int nb = aux_blocks(c, nc);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (mask_in)
    fallback_mask_kernel<true><<<nb, AUX_THREADS, 0, s>>>(trial_rho, mask_in, mask_out, g->nx, g->ny, g->nz);
  else
    fallback_mask_kernel<false><<<nb, AUX_THREADS, 0, s>>>(trial_rho, nullptr, mask_out, g->nx, g->ny, g->nz);
  PMF_CK(cudaGetLastError());
  return PMFMHD_OK;
}

}  // extern "C"
