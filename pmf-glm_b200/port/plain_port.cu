// The plain single-instance FP32 port of the reference's GLM step, for the benchmark only.
//
// A direct CUDA restatement of the reference's portable per-cell kernel as a GPU backend runs
// it (lib/MHDKernels/src/integrator_ref.jl:69-160, launched one thread per cell in groups of
// 256 by `_launch_step_ref!`, :189-201): every thread loads its own stencil from global
// memory, computes the Hancock prediction of its cell and of its six neighbours (seven
// `_mh_edges` calls) and solves its six faces, so each interior face is solved twice and each
// prediction repeated seven times. Periodic boundaries. Two arithmetics: the library's own
// (physics.cuh: packed FP32 pairs, the three-instruction MonCen), so that the comparison with
// the fused step kernel measures the decomposition alone (`pmfport_step_glm`), and the
// reference's scalar forms as a direct port compiles them (ref_arith.cuh,
// `pmfport_step_glm_refarith`). Not part of libpmfmhd.so: bench.py loads it as the "plain FP32
// port" baseline.
#include <cuda_runtime.h>

#include "../../include/pmfmhd.h"
#include "../csrc/physics.cuh"
#include "ref_arith.cuh"

namespace {

using namespace pmf;

struct PortArgs {
  const float* U[9];
  float* Un[9];
  int nx, ny, nz;
  float dtdx, ch, ich, decay;
  Phys P;
};

__device__ __forceinline__ int wrap(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// Primitive state of cell (i, j, k) (periodic images), glm_physics.jl:11-18.
__device__ __forceinline__ F9 load_prim(const PortArgs& a, int i, int j, int k) {
  const long long c = ((long long)wrap(k, a.nz) * a.ny + wrap(j, a.ny)) * a.nx + wrap(i, a.nx);
  F9 u;
#pragma unroll
  for (int f = 0; f < 9; ++f) u[f] = __ldg(a.U[f] + c);
  return cons2prim(u, a.P.gamma, a.P.smallr, a.P.pfl);
}

// `_mh_edges` (integrator_ref.jl:17-26) of cell (i, j, k): the Hancock-predicted primitive mh
// and the MC-PLM offsets of the three axes (REF: the reference's scalar arithmetic).
struct Edges {
  F9 mh;
  Offsets<RECON_PLM> o[3];
};
template <bool REF>
__device__ __forceinline__ Edges mh_edges(const PortArgs& a, int i, int j, int k) {
  Edges e;
  const F9 m0 = load_prim(a, i, j, k);
  if constexpr (REF) {
    e.o[0].dR = refarith::plm_slope(load_prim(a, i - 1, j, k), m0, load_prim(a, i + 1, j, k));
    e.o[1].dR = refarith::plm_slope(load_prim(a, i, j - 1, k), m0, load_prim(a, i, j + 1, k));
    e.o[2].dR = refarith::plm_slope(load_prim(a, i, j, k - 1), m0, load_prim(a, i, j, k + 1));
    e.mh = cons2prim(refarith::hancock_ref(m0, e.o[0].dR, e.o[1].dR, e.o[2].dR, a.dtdx, a.P.gamma), a.P.gamma,
                     a.P.smallr, a.P.pfl);
    return e;
  }
  e.o[0] = recon<RECON_PLM>(load_prim(a, i - 1, j, k), m0, load_prim(a, i + 1, j, k));
  e.o[1] = recon<RECON_PLM>(load_prim(a, i, j - 1, k), m0, load_prim(a, i, j + 1, k));
  e.o[2] = recon<RECON_PLM>(load_prim(a, i, j, k - 1), m0, load_prim(a, i, j, k + 1));
  const F9 u0 = prim2cons(m0, a.P.gamma);
  F9 acc = hancock_term<0, RECON_PLM>(m0, e.o[0], a.P.gamma);
  acc = add9(acc, hancock_term<1, RECON_PLM>(m0, e.o[1], a.P.gamma));
  acc = add9(acc, hancock_term<2, RECON_PLM>(m0, e.o[2], a.P.gamma));
  const float h = 0.5f * a.dtdx;
  F9 uh;
#pragma unroll
  for (int v = 0; v < 9; ++v) uh[v] = u0[v] - h * acc[v];
  e.mh = cons2prim(uh, a.P.gamma, a.P.smallr, a.P.pfl);
  return e;
}

template <int D, bool REF>
__device__ __forceinline__ F9 solve(const PortArgs& a, const F9& L, const F9& R) {
  if constexpr (REF) return refarith::riemann_ref<D>(L, R, a.ch, a.P);
  else return riemann<D, RS_HLLD, false>(L, R, a.ch, a.ich, a.P);
}

// Lower and upper D-faces of the cell: its neighbours' predictions recomputed, two solves.
template <int D, bool REF>
__device__ __forceinline__ void axis_fluxes(const PortArgs& a, int i, int j, int k, const Edges& ec, F9& Fl, F9& Fh) {
  const int di = D == 0, dj = D == 1, dk = D == 2;
  {
    const Edges em = mh_edges<REF>(a, i - di, j - dj, k - dk);
    Fl = solve<D, REF>(a, face_hi<RECON_PLM>(em.mh, em.o[D]), face_lo<RECON_PLM>(ec.mh, ec.o[D]));
  }
  {
    const Edges ep = mh_edges<REF>(a, i + di, j + dj, k + dk);
    Fh = solve<D, REF>(a, face_hi<RECON_PLM>(ec.mh, ec.o[D]), face_lo<RECON_PLM>(ep.mh, ep.o[D]));
  }
}

template <bool REF>
__global__ void __launch_bounds__(256) plain_port_kernel(const __grid_constant__ PortArgs a) {
  const long long c = (long long)blockIdx.x * 256 + threadIdx.x;
  const long long nc = (long long)a.nx * a.ny * a.nz;
  if (c >= nc) return;
  const int i = (int)(c % a.nx), j = (int)((c / a.nx) % a.ny), k = (int)(c / ((long long)a.nx * a.ny));
  const Edges ec = mh_edges<REF>(a, i, j, k);
  F9 div;
  {
    F9 Fl, Fh;
    axis_fluxes<0, REF>(a, i, j, k, ec, Fl, Fh);
#pragma unroll
    for (int v = 0; v < 9; ++v) div[v] = Fl[v] - Fh[v];
    axis_fluxes<1, REF>(a, i, j, k, ec, Fl, Fh);
#pragma unroll
    for (int v = 0; v < 9; ++v) div[v] = div[v] + (Fl[v] - Fh[v]);
    axis_fluxes<2, REF>(a, i, j, k, ec, Fl, Fh);
#pragma unroll
    for (int v = 0; v < 9; ++v) div[v] = div[v] + (Fl[v] - Fh[v]);
  }
#pragma unroll
  for (int v = 0; v < 8; ++v) a.Un[v][c] = __ldg(a.U[v] + c) + a.dtdx * div[v];
  a.Un[8][c] = (__ldg(a.U[8] + c) + a.dtdx * div[8]) * a.decay;
}

template <bool REF>
int port_step(const pmfmhd_grid* g, const float* const U[9], float* const Unew[9], float dt, float ch, float decay,
              void* stream) {
  if (g == nullptr || U == nullptr || Unew == nullptr) return PMFMHD_EINVAL;
  if (g->nx < 1 || g->ny < 1 || g->nz < 1) return PMFMHD_ESHAPE;
  if (g->recon != PMFMHD_RECON_PLM || g->riemann != PMFMHD_RIEMANN_HLLD) return PMFMHD_EUNSUPPORTED;
  for (int d = 0; d < 3; ++d)
    if (g->bc[d] != PMFMHD_BC_PERIODIC) return PMFMHD_EUNSUPPORTED;
  PortArgs a;
  for (int f = 0; f < 9; ++f) {
    if (U[f] == nullptr || Unew[f] == nullptr) return PMFMHD_EINVAL;
    a.U[f] = U[f];
    a.Un[f] = Unew[f];
  }
  a.nx = g->nx; a.ny = g->ny; a.nz = g->nz;
  a.dtdx = dt / g->dx; a.ch = ch; a.ich = 1.0f / ch; a.decay = decay;
  a.P = Phys{g->gamma, g->smallr, g->pfl, g->llf_dmin, g->llf_pmin, g->hlld_dtol_rel};
  const long long nc = (long long)g->nx * g->ny * g->nz;
  plain_port_kernel<REF><<<(unsigned)((nc + 255) / 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(a);
  return cudaGetLastError() == cudaSuccess ? PMFMHD_OK : PMFMHD_ECUDA;
}

}  // namespace

// One plain GLM step (MC-PLM, HLLD, all-periodic) of the grid `g`: U in, Unew out, on `stream`,
// with the library's arithmetic. Returns 0, or a negative PMFMHD_E* code for arguments the
// port does not cover.
extern "C" int pmfport_step_glm(const pmfmhd_grid* g, const float* const U[9], float* const Unew[9], float dt,
                                float ch, float decay, void* stream) {
  return port_step<false>(g, U, Unew, dt, ch, decay, stream);
}
// The same step with the reference's scalar arithmetic (glm_physics.jl forms).
extern "C" int pmfport_step_glm_refarith(const pmfmhd_grid* g, const float* const U[9], float* const Unew[9],
                                         float dt, float ch, float decay, void* stream) {
  return port_step<true>(g, U, Unew, dt, ch, decay, stream);
}
