// Cell-local linear drag operators of the split drag steps (lib/MHDKernels/src/drag.jl):
//   pmfmhd_apply_linear_drag                 <- apply_linear_drag!                (drag.jl:78-117)
//   pmfmhd_apply_exponential_drag_increment  <- apply_exponential_drag_increment! (drag.jl:121-208)
// Both are one pass over the cells (HBM-bound: 36 B/cell and 60 B/cell); the per-step
// coefficients exp(-q) and phi1(q) are computed once on the host in FP32.
#include <cmath>

#include "aux_kernels.cuh"
#include "host_internal.h"

namespace pmf {
namespace {

struct Vel3 {
  float x, y, z;
};

// Exact constant-coefficient drag over an interval with velocity decay factor `decay`;
// the kinetic energy removed is removed from E (optionally Kahan-compensated).
template <bool COMP>
__global__ void __launch_bounds__(AUX_THREADS) linear_drag_kernel(float* __restrict__ mx, float* __restrict__ my,
                                                                  float* __restrict__ mz, float* __restrict__ E,
                                                                  const float* __restrict__ rho,
                                                                  float* __restrict__ eres, long long nc, Vel3 v0,
                                                                  float decay, float smallr, float smallE) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < nc; c += (long long)gridDim.x * blockDim.x) {
    const float r = fmaxf(rho[c], smallr);
    const float ox = mx[c], oy = my[c], oz = mz[c];
    const float tx = r * v0.x, ty = r * v0.y, tz = r * v0.z;
    const float ek0 = 0.5f * (ox * ox + oy * oy + oz * oz) / r;
    const float nx = tx + (ox - tx) * decay, ny = ty + (oy - ty) * decay, nz = tz + (oz - tz) * decay;
    const float ek1 = 0.5f * (nx * nx + ny * ny + nz * nz) / r;
    mx[c] = nx;
    my[c] = ny;
    mz[c] = nz;
    float e;
    if constexpr (COMP) {
      float rr = eres[c];
      e = comp_add(E[c], ek1 - ek0, rr);
      eres[c] = rr;
    } else {
      e = E[c] + (ek1 - ek0);
    }
    E[c] = fmaxf(e, smallE);
  }
}

// Exponential constant-force update of a no-drag trial (s.U) given the state before it.
__global__ void __launch_bounds__(AUX_THREADS) exp_drag_increment_kernel(
    float* __restrict__ mx, float* __restrict__ my, float* __restrict__ mz, float* __restrict__ E,
    const float* __restrict__ rho, const float* __restrict__ orho, const float* __restrict__ omx,
    const float* __restrict__ omy, const float* __restrict__ omz, const float* __restrict__ bx,
    const float* __restrict__ by, const float* __restrict__ bz, long long nc, Vel3 v0, float decay, float phi1,
    float smallr, float smallE) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < nc; c += (long long)gridDim.x * blockDim.x) {
    const float rn = fmaxf(rho[c], smallr), ro = fmaxf(orho[c], smallr);
    const float tmx = mx[c], tmy = my[c], tmz = mz[c];
    const float vox = omx[c] / ro, voy = omy[c] / ro, voz = omz[c] / ro;
    const float vtx = tmx / rn, vty = tmy / rn, vtz = tmz / rn;
    const float ek0 = 0.5f * (tmx * tmx + tmy * tmy + tmz * tmz) / rn;
    const float b1 = bx[c], b2 = by[c], b3 = bz[c];
    const float eb = 0.5f * (b1 * b1 + b2 * b2 + b3 * b3);
    const float nonkinetic = fmaxf(E[c] - ek0, eb + smallE);
    const float vnx = v0.x + decay * (vox - v0.x) + phi1 * (vtx - vox);
    const float vny = v0.y + decay * (voy - v0.y) + phi1 * (vty - voy);
    const float vnz = v0.z + decay * (voz - v0.z) + phi1 * (vtz - voz);
    const float nmx = rn * vnx, nmy = rn * vny, nmz = rn * vnz;
    const float ek1 = 0.5f * (nmx * nmx + nmy * nmy + nmz * nmz) / rn;
    mx[c] = nmx;
    my[c] = nmy;
    mz[c] = nmz;
    E[c] = fmaxf(nonkinetic + ek1, eb + smallE);
  }
}

Vel3 vel3(const float* v) { return v ? Vel3{v[0], v[1], v[2]} : Vel3{0.0f, 0.0f, 0.0f}; }

}  // namespace
}  // namespace pmf

using namespace pmf;
using namespace pmf::host;

extern "C" {

int pmfmhd_apply_linear_drag(pmfmhd_ctx* c, const pmfmhd_grid* g, float* const U[9], float decay,
                             const float target_velocity[3], float* energy_residual, void* stream) {
  if (c == nullptr || U == nullptr) return PMFMHD_EINVAL;
  int rc = check_grid(g);
  if (rc) return rc;
  for (int f = 0; f < 5; ++f)
    if (U[f] == nullptr) return PMFMHD_EINVAL;
  if (!std::isfinite(decay) || decay < 0.0f || decay > 1.0f) return PMFMHD_EINVAL;
  const long long nc = ncells(g);
  const int nb = aux_blocks(c, nc);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (energy_residual)
    linear_drag_kernel<true><<<nb, AUX_THREADS, 0, s>>>(U[1], U[2], U[3], U[4], U[0], energy_residual, nc,
                                                        vel3(target_velocity), decay, g->smallr, 1e-30f);
  else
    linear_drag_kernel<false><<<nb, AUX_THREADS, 0, s>>>(U[1], U[2], U[3], U[4], U[0], nullptr, nc,
                                                         vel3(target_velocity), decay, g->smallr, 1e-30f);
  PMF_CK(cudaGetLastError());
  return PMFMHD_OK;
}

int pmfmhd_apply_exponential_drag_increment(pmfmhd_ctx* c, const pmfmhd_grid* g, float* const U[9],
                                            const float* const old_U[9], float drag_impulse,
                                            const float target_velocity[3], void* stream) {
  if (c == nullptr || U == nullptr || old_U == nullptr) return PMFMHD_EINVAL;
  int rc = check_grid(g);
  if (rc) return rc;
  for (int f = 0; f < 8; ++f)
    if (U[f] == nullptr || (f < 4 && old_U[f] == nullptr)) return PMFMHD_EINVAL;
  if (!std::isfinite(drag_impulse) || !(drag_impulse >= 0.0f)) return PMFMHD_EINVAL;
  const DragCoef k = drag_coefficients(drag_impulse, target_velocity);
  const long long nc = ncells(g);
  const int nb = aux_blocks(c, nc);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  exp_drag_increment_kernel<<<nb, AUX_THREADS, 0, s>>>(U[1], U[2], U[3], U[4], U[0], old_U[0], old_U[1], old_U[2],
                                                      old_U[3], U[5], U[6], U[7], nc, vel3(target_velocity), k.decay,
                                                      k.phi1, g->smallr, 1e-30f);
  PMF_CK(cudaGetLastError());
  return PMFMHD_OK;
}

}  // extern "C"
