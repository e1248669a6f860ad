// Terminal-regime induction (lib/MHDKernels/src/terminal_ct.jl): in the overdamped early-PMF
// regime the gas velocity is the terminal velocity v = (F_Maxwell - c_p grad rho) / (rho Gamma)
// and only the induction equation is advanced, by SSPRK2 with a centred curl (GLM states) or
// the edge-averaged face curl (CT states), plus order-2 or order-4 dissipation.
//
//   pmfmhd_terminal_magnetic_force        <- terminal_magnetic_force!       (terminal_ct.jl:99-106)
//   pmfmhd_terminal_magnetic_force_split  <- terminal_magnetic_force_split! (:117-126)
//   pmfmhd_terminal_velocity_max          <- terminal_velocity_max!         (:226-238)
//   pmfmhd_terminal_ct_induction          <- terminal_ct_induction!         (:502-575)
//   pmfmhd_terminal_ct_euler_from_cell_emf <- terminal_ct_euler_from_cell_emf! (:461-486)
//
// Design: the reference recomputes the terminal EMF of each of a cell's six neighbours inside
// its update kernel (the Maxwell force at the neighbour is an array, the velocity and v x B are
// recomputed per use). Here one kernel computes the Maxwell force, the terminal velocity and
// e = v x B once per cell (the values are the same, computed from the same inputs), and the
// stage kernel takes the curl of that EMF field: two passes per SSPRK2 stage instead of
// three, and 1/6 of the velocity work. Every grid is cubic and periodic.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>

#include "aux_kernels.cuh"
#include "host_internal.h"

namespace pmf {
namespace {

constexpr int kT = 256;

struct Cube {
  int N;
  __device__ __forceinline__ long long at(int i, int j, int k) const {
    i = (i + 2 * N) % N;
    j = (j + 2 * N) % N;
    k = (k + 2 * N) % N;
    return ((long long)k * N + j) * N + i;
  }
  __device__ __forceinline__ void ijk(long long c, int& i, int& j, int& k) const {
    i = (int)(c % N);
    j = (int)((c / N) % N);
    k = (int)(c / ((long long)N * N));
  }
};

struct F3 {
  float x, y, z;
};

// Conservative centred Maxwell-stress divergence (terminal_ct.jl:18-51)
__device__ __forceinline__ F3 maxwell_force(const float* __restrict__ bx, const float* __restrict__ by,
                                            const float* __restrict__ bz, const Cube& G, int i, int j, int k,
                                            float inv2dx) {
  float t[3][3];  // t[component][direction]
  const int o[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const long long p = G.at(i + o[d][0], j + o[d][1], k + o[d][2]);
    const long long m = G.at(i - o[d][0], j - o[d][1], k - o[d][2]);
    const float bp[3] = {bx[p], by[p], bz[p]}, bm[3] = {bx[m], by[m], bz[m]};
    const float b2p = bp[0] * bp[0] + bp[1] * bp[1] + bp[2] * bp[2];
    const float b2m = bm[0] * bm[0] + bm[1] * bm[1] + bm[2] * bm[2];
#pragma unroll
    for (int c = 0; c < 3; ++c)
      t[c][d] = c == d ? (bp[c] * bp[c] - 0.5f * b2p) - (bm[c] * bm[c] - 0.5f * b2m) : bp[c] * bp[d] - bm[c] * bm[d];
  }
  return F3{(t[0][0] + t[0][1] + t[0][2]) * inv2dx, (t[1][0] + t[1][1] + t[1][2]) * inv2dx,
            (t[2][0] + t[2][1] + t[2][2]) * inv2dx};
}

struct Terminal {
  float inv2dx, gamma_drag, pressure_coeff, smallr, vcap;
};

// Terminal velocity (terminal_ct.jl:125-145), capped at vcap
__device__ __forceinline__ F3 terminal_velocity(const float* __restrict__ rho, F3 f, const Cube& G, long long c, int i,
                                                int j, int k, const Terminal& P) {
  const float r = fmaxf(rho[c], P.smallr);
  const float gx = P.pressure_coeff * (rho[G.at(i + 1, j, k)] - rho[G.at(i - 1, j, k)]) * P.inv2dx;
  const float gy = P.pressure_coeff * (rho[G.at(i, j + 1, k)] - rho[G.at(i, j - 1, k)]) * P.inv2dx;
  const float gz = P.pressure_coeff * (rho[G.at(i, j, k + 1)] - rho[G.at(i, j, k - 1)]) * P.inv2dx;
  const float invrg = 1.0f / (r * fmaxf(P.gamma_drag, FLT_EPSILON));
  F3 v{(f.x - gx) * invrg, (f.y - gy) * invrg, (f.z - gz) * invrg};
  const float v2 = v.x * v.x + v.y * v.y + v.z * v.z;
  if (v2 > P.vcap * P.vcap) {
    const float q = P.vcap / sqrtf(v2);
    v.x *= q;
    v.y *= q;
    v.z *= q;
  }
  return v;
}

__global__ void __launch_bounds__(kT) force_kernel(const float* __restrict__ bx, const float* __restrict__ by,
                                                   const float* __restrict__ bz, float* __restrict__ fx,
                                                   float* __restrict__ fy, float* __restrict__ fz,
                                                   float* __restrict__ px, float* __restrict__ py,
                                                   float* __restrict__ pz, Cube G, float inv2dx) {
  const long long n = (long long)G.N * G.N * G.N;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    G.ijk(c, i, j, k);
    const F3 f = maxwell_force(bx, by, bz, G, i, j, k, inv2dx);
    if (px == nullptr) {
      fx[c] = f.x;
      fy[c] = f.y;
      fz[c] = f.z;
      continue;
    }
    // split (terminal_ct.jl:53-69): pressure -grad(B^2/2), tension = remainder (into f*)
    auto b2 = [&](long long q) { return bx[q] * bx[q] + by[q] * by[q] + bz[q] * bz[q]; };
    const float ppx = -0.5f * (b2(G.at(i + 1, j, k)) - b2(G.at(i - 1, j, k))) * inv2dx;
    const float ppy = -0.5f * (b2(G.at(i, j + 1, k)) - b2(G.at(i, j - 1, k))) * inv2dx;
    const float ppz = -0.5f * (b2(G.at(i, j, k + 1)) - b2(G.at(i, j, k - 1))) * inv2dx;
    px[c] = ppx;
    py[c] = ppy;
    pz[c] = ppz;
    fx[c] = f.x - ppx;
    fy[c] = f.y - ppy;
    fz[c] = f.z - ppz;
  }
}

// Cell EMF e = v x B with the terminal velocity of the field (bx, by, bz); optional running
// maximum of |v| (bits of a non-negative float).
__global__ void __launch_bounds__(kT) cell_emf_kernel(const float* __restrict__ rho, const float* __restrict__ bx,
                                                      const float* __restrict__ by, const float* __restrict__ bz,
                                                      float* __restrict__ ex, float* __restrict__ ey,
                                                      float* __restrict__ ez, unsigned int* __restrict__ vmax_bits,
                                                      Cube G, Terminal P) {
  const long long n = (long long)G.N * G.N * G.N;
  float vm = 0.0f;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    G.ijk(c, i, j, k);
    const F3 f = maxwell_force(bx, by, bz, G, i, j, k, P.inv2dx);
    const F3 v = terminal_velocity(rho, f, G, c, i, j, k, P);
    if (vmax_bits != nullptr) {
      vm = fmaxf(vm, sqrtf(v.x * v.x + v.y * v.y + v.z * v.z));
    } else {
      const float b1 = bx[c], b2 = by[c], b3 = bz[c];
      ex[c] = v.y * b3 - v.z * b2;
      ey[c] = v.z * b1 - v.x * b3;
      ez[c] = v.x * b2 - v.y * b1;
    }
  }
  if (vmax_bits != nullptr) {
    vm = warp_max(vm);
    if ((threadIdx.x & 31) == 0) atomicMax(vmax_bits, __float_as_uint(vm));
  }
}

__device__ __forceinline__ float lap(const float* __restrict__ A, const Cube& G, int i, int j, int k, float invdx2) {
  const float s = A[G.at(i + 1, j, k)] + A[G.at(i - 1, j, k)] + A[G.at(i, j + 1, k)] + A[G.at(i, j - 1, k)] +
                  A[G.at(i, j, k + 1)] + A[G.at(i, j, k - 1)];
  return (s - 6.0f * A[G.at(i, j, k)]) * invdx2;
}

// 25-point bilaplacian (terminal_ct.jl:166-181)
__device__ __forceinline__ float bilap(const float* __restrict__ A, const Cube& G, int i, int j, int k, float invdx2) {
  const float c = A[G.at(i, j, k)];
  const float a1 = A[G.at(i + 1, j, k)] + A[G.at(i - 1, j, k)] + A[G.at(i, j + 1, k)] + A[G.at(i, j - 1, k)] +
                   A[G.at(i, j, k + 1)] + A[G.at(i, j, k - 1)];
  const float a2 = A[G.at(i + 2, j, k)] + A[G.at(i - 2, j, k)] + A[G.at(i, j + 2, k)] + A[G.at(i, j - 2, k)] +
                   A[G.at(i, j, k + 2)] + A[G.at(i, j, k - 2)];
  const float dg = A[G.at(i + 1, j + 1, k)] + A[G.at(i + 1, j - 1, k)] + A[G.at(i - 1, j + 1, k)] +
                   A[G.at(i - 1, j - 1, k)] + A[G.at(i + 1, j, k + 1)] + A[G.at(i + 1, j, k - 1)] +
                   A[G.at(i - 1, j, k + 1)] + A[G.at(i - 1, j, k - 1)] + A[G.at(i, j + 1, k + 1)] +
                   A[G.at(i, j + 1, k - 1)] + A[G.at(i, j - 1, k + 1)] + A[G.at(i, j - 1, k - 1)];
  return ((42.0f * c - 12.0f * a1) + a2 + 2.0f * dg) * invdx2 * invdx2;
}

__device__ __forceinline__ float dissip(const float* __restrict__ A, const Cube& G, int i, int j, int k, float invdx2,
                                        float eta, int order) {
  return order == 4 ? -eta * bilap(A, G, i, j, k, invdx2) : eta * lap(A, G, i, j, k, invdx2);
}

struct Stage {
  float dt, inv2dx, invdx, invdx2, eta;
  int order;
};

// GLM SSPRK2 stage (terminal_ct.jl:240-293). stage 0: out = B + dt*rhs(e, B).
// stage 1: B <- (B + pB + dt*rhs(e, pB))/2 in place, E follows the magnetic energy.
__global__ void __launch_bounds__(kT) glm_stage_kernel(const float* __restrict__ ex, const float* __restrict__ ey,
                                                       const float* __restrict__ ez, float* bx, float* by, float* bz,
                                                       float* __restrict__ pbx, float* __restrict__ pby,
                                                       float* __restrict__ pbz, float* __restrict__ E, Cube G, Stage S,
                                                       int stage) {
  const long long n = (long long)G.N * G.N * G.N;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    G.ijk(c, i, j, k);
    const float cx = ((ez[G.at(i, j + 1, k)] - ez[G.at(i, j - 1, k)]) - (ey[G.at(i, j, k + 1)] - ey[G.at(i, j, k - 1)])) *
                     S.inv2dx;
    const float cy = ((ex[G.at(i, j, k + 1)] - ex[G.at(i, j, k - 1)]) - (ez[G.at(i + 1, j, k)] - ez[G.at(i - 1, j, k)])) *
                     S.inv2dx;
    const float cz = ((ey[G.at(i + 1, j, k)] - ey[G.at(i - 1, j, k)]) - (ex[G.at(i, j + 1, k)] - ex[G.at(i, j - 1, k)])) *
                     S.inv2dx;
    if (stage == 0) {
      pbx[c] = bx[c] + S.dt * (cx + dissip(bx, G, i, j, k, S.invdx2, S.eta, S.order));
      pby[c] = by[c] + S.dt * (cy + dissip(by, G, i, j, k, S.invdx2, S.eta, S.order));
      pbz[c] = bz[c] + S.dt * (cz + dissip(bz, G, i, j, k, S.invdx2, S.eta, S.order));
    } else {
      const float rx = cx + dissip(pbx, G, i, j, k, S.invdx2, S.eta, S.order);
      const float ry = cy + dissip(pby, G, i, j, k, S.invdx2, S.eta, S.order);
      const float rz = cz + dissip(pbz, G, i, j, k, S.invdx2, S.eta, S.order);
      const float ox = bx[c], oy = by[c], oz = bz[c];
      const float nx = 0.5f * ((ox + pbx[c]) + S.dt * rx);
      const float ny = 0.5f * ((oy + pby[c]) + S.dt * ry);
      const float nz = 0.5f * ((oz + pbz[c]) + S.dt * rz);
      const float eb0 = 0.5f * (ox * ox + oy * oy + oz * oz);
      const float eb1 = 0.5f * (nx * nx + ny * ny + nz * nz);
      bx[c] = nx;
      by[c] = ny;
      bz[c] = nz;
      E[c] = fmaxf((E[c] + eb1) - eb0, 1e-30f);
    }
  }
}

// Edge EMF = mean of the four cells sharing the edge (terminal_ct.jl:325-345)
__global__ void __launch_bounds__(kT) edge_kernel(const float* __restrict__ ecx, const float* __restrict__ ecy,
                                                  const float* __restrict__ ecz, float* __restrict__ ex,
                                                  float* __restrict__ ey, float* __restrict__ ez, Cube G) {
  const long long n = (long long)G.N * G.N * G.N;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    G.ijk(c, i, j, k);
    const long long im = G.at(i - 1, j, k), jm = G.at(i, j - 1, k), km = G.at(i, j, k - 1);
    ez[c] = 0.25f * (((ecz[c] + ecz[im]) + ecz[jm]) + ecz[G.at(i - 1, j - 1, k)]);
    ex[c] = 0.25f * (((ecx[c] + ecx[jm]) + ecx[km]) + ecx[G.at(i, j - 1, k - 1)]);
    ey[c] = 0.25f * (((ecy[c] + ecy[im]) + ecy[km]) + ecy[G.at(i - 1, j, k - 1)]);
  }
}

// CT SSPRK2 stage on the faces (terminal_ct.jl:347-407). stage 0: pf = f + dt*rate(e, f).
// stage 1: f <- (f + pf + dt*rate(e, pf))/2 in place, Kahan-compensated when `comp`.
__global__ void __launch_bounds__(kT) face_stage_kernel(const float* __restrict__ ex, const float* __restrict__ ey,
                                                        const float* __restrict__ ez, float* fx, float* fy, float* fz,
                                                        float* __restrict__ pfx, float* __restrict__ pfy,
                                                        float* __restrict__ pfz, float* __restrict__ rbx,
                                                        float* __restrict__ rby, float* __restrict__ rbz, Cube G,
                                                        Stage S, int stage, int comp) {
  const long long n = (long long)G.N * G.N * G.N;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    G.ijk(c, i, j, k);
    const long long ip = G.at(i + 1, j, k), jp = G.at(i, j + 1, k), kp = G.at(i, j, k + 1);
    const float cx = ((ez[jp] - ez[c]) - (ey[kp] - ey[c])) * S.invdx;
    const float cy = ((ex[kp] - ex[c]) - (ez[ip] - ez[c])) * S.invdx;
    const float cz = ((ey[ip] - ey[c]) - (ex[jp] - ex[c])) * S.invdx;
    if (stage == 0) {
      pfx[c] = fx[c] + S.dt * (cx + dissip(fx, G, i, j, k, S.invdx2, S.eta, S.order));
      pfy[c] = fy[c] + S.dt * (cy + dissip(fy, G, i, j, k, S.invdx2, S.eta, S.order));
      pfz[c] = fz[c] + S.dt * (cz + dissip(fz, G, i, j, k, S.invdx2, S.eta, S.order));
    } else {
      const float x = cx + dissip(pfx, G, i, j, k, S.invdx2, S.eta, S.order);
      const float y = cy + dissip(pfy, G, i, j, k, S.invdx2, S.eta, S.order);
      const float z = cz + dissip(pfz, G, i, j, k, S.invdx2, S.eta, S.order);
      const float ox = fx[c], oy = fy[c], oz = fz[c];
      if (comp) {
        float r1 = rbx[c], r2 = rby[c], r3 = rbz[c];
        fx[c] = comp_add(ox, 0.5f * ((pfx[c] - ox) + S.dt * x), r1);
        fy[c] = comp_add(oy, 0.5f * ((pfy[c] - oy) + S.dt * y), r2);
        fz[c] = comp_add(oz, 0.5f * ((pfz[c] - oz) + S.dt * z), r3);
        rbx[c] = r1;
        rby[c] = r2;
        rbz[c] = r3;
      } else {
        fx[c] = 0.5f * ((ox + pfx[c]) + S.dt * x);
        fy[c] = 0.5f * ((oy + pfy[c]) + S.dt * y);
        fz[c] = 0.5f * ((oz + pfz[c]) + S.dt * z);
      }
    }
  }
}

// Face average into cell B; with E, E follows the magnetic-energy change (floor smallE)
// (terminal_ct.jl:409-427, ct.jl:205-219 `_ct_bcc_k!` without E).
__global__ void __launch_bounds__(kT) face_average_kernel(const float* __restrict__ fx, const float* __restrict__ fy,
                                                          const float* __restrict__ fz, float* __restrict__ bx,
                                                          float* __restrict__ by, float* __restrict__ bz,
                                                          float* __restrict__ E, float* __restrict__ psi, Cube G,
                                                          int energy_mode) {
  const long long n = (long long)G.N * G.N * G.N;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    G.ijk(c, i, j, k);
    const float nx = 0.5f * (fx[c] + fx[G.at(i + 1, j, k)]);
    const float ny = 0.5f * (fy[c] + fy[G.at(i, j + 1, k)]);
    const float nz = 0.5f * (fz[c] + fz[G.at(i, j, k + 1)]);
    if (energy_mode != 0) {
      const float ox = bx[c], oy = by[c], oz = bz[c];
      if (energy_mode == 1) {  // terminal corrector: E += eb1 - eb0, floored
        const float eb0 = 0.5f * (ox * ox + oy * oy + oz * oz);
        const float eb1 = 0.5f * (nx * nx + ny * ny + nz * nz);
        E[c] = fmaxf((E[c] + eb1) - eb0, 1e-30f);
      } else {  // face install: E += (|B_new|^2 - |B_old|^2)/2, psi = 0
        E[c] += 0.5f * ((nx * nx + ny * ny + nz * nz) - (ox * ox + oy * oy + oz * oz));
        psi[c] = 0.0f;
      }
    }
    bx[c] = nx;
    by[c] = ny;
    bz[c] = nz;
  }
}

// Forward-Euler compensated face update from edge EMFs (terminal_ct.jl:461-474)
__global__ void __launch_bounds__(kT) face_euler_kernel(float* fx, float* fy, float* fz, float* rbx, float* rby,
                                                        float* rbz, const float* __restrict__ ex,
                                                        const float* __restrict__ ey, const float* __restrict__ ez,
                                                        Cube G, float dt, float invdx) {
  const long long n = (long long)G.N * G.N * G.N;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    G.ijk(c, i, j, k);
    const long long ip = G.at(i + 1, j, k), jp = G.at(i, j + 1, k), kp = G.at(i, j, k + 1);
    float r1 = rbx[c], r2 = rby[c], r3 = rbz[c];
    fx[c] = comp_add(fx[c], dt * ((ez[jp] - ez[c]) - (ey[kp] - ey[c])) * invdx, r1);
    fy[c] = comp_add(fy[c], dt * ((ex[kp] - ex[c]) - (ez[ip] - ez[c])) * invdx, r2);
    fz[c] = comp_add(fz[c], dt * ((ey[ip] - ey[c]) - (ex[jp] - ex[c])) * invdx, r3);
    rbx[c] = r1;
    rby[c] = r2;
    rbz[c] = r3;
  }
}

int cube_of(const pmfmhd_grid* g, Cube* G) {
  if (g->nx != g->ny || g->nx != g->nz) return PMFMHD_ESHAPE;  // terminal CT requires a cubic grid
  if (!(g->bc[0] == PMFMHD_BC_PERIODIC && g->bc[1] == PMFMHD_BC_PERIODIC && g->bc[2] == PMFMHD_BC_PERIODIC))
    return PMFMHD_EUNSUPPORTED;
  G->N = g->nx;
  return PMFMHD_OK;
}

}  // namespace
}  // namespace pmf

using namespace pmf;
using namespace pmf::host;

extern "C" {

int pmfmhd_terminal_magnetic_force(pmfmhd_ctx* c, const pmfmhd_grid* g, const float* const B[3], float* const F[3],
                                   float* const P[3], void* stream) {
  if (c == nullptr || B == nullptr || F == nullptr) return PMFMHD_EINVAL;
  int rc = check_grid(g);
  if (rc) return rc;
  Cube G;
  if ((rc = cube_of(g, &G))) return rc;
  for (int d = 0; d < 3; ++d)
    if (!B[d] || !F[d] || (P && !P[d])) return PMFMHD_EINVAL;
  const long long n = ncells(g);
  force_kernel<<<aux_blocks(c, n), kT, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      B[0], B[1], B[2], F[0], F[1], F[2], P ? P[0] : nullptr, P ? P[1] : nullptr, P ? P[2] : nullptr, G,
      1.0f / (2.0f * g->dx));
  PMF_CK(cudaGetLastError());
  return PMFMHD_OK;
}

int pmfmhd_terminal_velocity_max(pmfmhd_ctx* c, const pmfmhd_grid* g, const float* const U[9], float gamma_drag,
                                 float pressure_coeff, float vcap, double* vmax, void* stream) {
  if (c == nullptr || U == nullptr || vmax == nullptr || !U[0] || !U[5] || !U[6] || !U[7]) return PMFMHD_EINVAL;
  int rc = check_grid(g);
  if (rc) return rc;
  Cube G;
  if ((rc = cube_of(g, &G))) return rc;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const long long n = ncells(g);
  PMF_CK(cudaMemsetAsync(c->d_u64, 0, sizeof(unsigned int), s));
  Terminal P{1.0f / (2.0f * g->dx), gamma_drag, pressure_coeff, g->smallr, vcap};
  unsigned int* bits = reinterpret_cast<unsigned int*>(c->d_u64);
  cell_emf_kernel<<<aux_blocks(c, n), kT, 0, s>>>(U[0], U[5], U[6], U[7], nullptr, nullptr, nullptr, bits, G, P);
  PMF_CK(cudaGetLastError());
  unsigned int hb = 0;
  PMF_CK(cudaMemcpyAsync(c->h_pin, bits, sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
  PMF_CK(cudaStreamSynchronize(s));
  std::memcpy(&hb, c->h_pin, sizeof(hb));
  float v;
  std::memcpy(&v, &hb, sizeof(v));
  *vmax = (double)v;
  return PMFMHD_OK;
}

int pmfmhd_terminal_ct_induction(pmfmhd_ctx* c, const pmfmhd_grid* g, float* const U[9], float* const scratch[9],
                                 float* ct, float dt, float gamma_drag, float pressure_coeff, float cfl,
                                 float dissipation, int dissipation_order, float vcap, int max_subcycles,
                                 int compensate, int* nsub_out, double* vmax_out, double* eta_out, void* stream) {
  if (c == nullptr || U == nullptr || scratch == nullptr) return PMFMHD_EINVAL;
  int rc = check_grid(g);
  if (rc) return rc;
  Cube G;
  if ((rc = cube_of(g, &G))) return rc;
  for (int f = 0; f < 9; ++f)
    if (!U[f] || !scratch[f]) return PMFMHD_EINVAL;
  if (!(cfl > 0.0f && cfl <= 1.0f) || !(dissipation >= 0.0f && dissipation <= 1.0f)) return PMFMHD_EINVAL;
  if (dissipation_order != 2 && dissipation_order != 4) return PMFMHD_EINVAL;
  if (!std::isfinite(dt) || !std::isfinite(gamma_drag) || !std::isfinite(pressure_coeff)) return PMFMHD_EINVAL;
  double vmax = 0.0;
  if ((rc = pmfmhd_terminal_velocity_max(c, g, U, gamma_drag, pressure_coeff, vcap, &vmax, stream))) return rc;
  const double dx = (double)g->dx;
  const long long nsub = std::max<long long>(
      1, (long long)std::ceil((double)dt * vmax / std::max((double)cfl * dx, DBL_EPSILON)));
  if (nsub > max_subcycles) return PMFMHD_EINADMISSIBLE;  // the caller's subcycle limit
  Stage S;
  S.dt = (float)((double)dt / (double)nsub);
  S.inv2dx = 1.0f / (2.0f * g->dx);
  S.invdx = 1.0f / g->dx;
  S.invdx2 = 1.0f / (g->dx * g->dx);
  S.eta = dissipation_order == 4 ? (float)(dissipation / 12.0) * (float)vmax * (g->dx * g->dx * g->dx)
                                 : dissipation * (float)vmax * g->dx;
  S.order = dissipation_order;
  Terminal P{S.inv2dx, gamma_drag, pressure_coeff, g->smallr, vcap};
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const long long n = ncells(g);
  const int nb = aux_blocks(c, n);
  for (long long it = 0; it < nsub; ++it) {
    if (ct == nullptr) {
      // GLM: cell EMF -> scratch[1..3], predictor -> scratch[5..7]
      cell_emf_kernel<<<nb, kT, 0, s>>>(U[0], U[5], U[6], U[7], scratch[1], scratch[2], scratch[3], nullptr, G, P);
      glm_stage_kernel<<<nb, kT, 0, s>>>(scratch[1], scratch[2], scratch[3], U[5], U[6], U[7], scratch[5], scratch[6],
                                         scratch[7], U[4], G, S, 0);
      cell_emf_kernel<<<nb, kT, 0, s>>>(U[0], scratch[5], scratch[6], scratch[7], scratch[1], scratch[2], scratch[3],
                                        nullptr, G, P);
      glm_stage_kernel<<<nb, kT, 0, s>>>(scratch[1], scratch[2], scratch[3], U[5], U[6], U[7], scratch[5], scratch[6],
                                         scratch[7], U[4], G, S, 1);
    } else {
      // CT: workspace in the packed buffer as the reference (cell EMF ec*, edge EMF e*,
      // predicted faces mf*), the predictor's cell B in scratch[5..7]
      auto slot = [&](int q) { return ct + (size_t)q * n; };
      cell_emf_kernel<<<nb, kT, 0, s>>>(U[0], U[5], U[6], U[7], slot(CT_ECX), slot(CT_ECY), slot(CT_ECZ), nullptr, G,
                                        P);
      edge_kernel<<<nb, kT, 0, s>>>(slot(CT_ECX), slot(CT_ECY), slot(CT_ECZ), slot(CT_EX), slot(CT_EY), slot(CT_EZ), G);
      face_stage_kernel<<<nb, kT, 0, s>>>(slot(CT_EX), slot(CT_EY), slot(CT_EZ), slot(CT_BXF), slot(CT_BYF),
                                          slot(CT_BZF), slot(CT_MFX), slot(CT_MFY), slot(CT_MFZ), nullptr, nullptr,
                                          nullptr, G, S, 0, 0);
      face_average_kernel<<<nb, kT, 0, s>>>(slot(CT_MFX), slot(CT_MFY), slot(CT_MFZ), scratch[5], scratch[6],
                                            scratch[7], nullptr, nullptr, G, 0);
      cell_emf_kernel<<<nb, kT, 0, s>>>(U[0], scratch[5], scratch[6], scratch[7], slot(CT_ECX), slot(CT_ECY),
                                        slot(CT_ECZ), nullptr, G, P);
      edge_kernel<<<nb, kT, 0, s>>>(slot(CT_ECX), slot(CT_ECY), slot(CT_ECZ), slot(CT_EX), slot(CT_EY), slot(CT_EZ), G);
      face_stage_kernel<<<nb, kT, 0, s>>>(slot(CT_EX), slot(CT_EY), slot(CT_EZ), slot(CT_BXF), slot(CT_BYF),
                                          slot(CT_BZF), slot(CT_MFX), slot(CT_MFY), slot(CT_MFZ), slot(CT_RBX),
                                          slot(CT_RBY), slot(CT_RBZ), G, S, 1, compensate);
      face_average_kernel<<<nb, kT, 0, s>>>(slot(CT_BXF), slot(CT_BYF), slot(CT_BZF), U[5], U[6], U[7], U[4], nullptr,
                                            G, 1);
    }
  }
  PMF_CK(cudaGetLastError());
  if (nsub_out) *nsub_out = (int)nsub;
  if (vmax_out) *vmax_out = vmax;
  if (eta_out) *eta_out = (double)S.eta;
  return PMFMHD_OK;
}

int pmfmhd_terminal_ct_euler_from_cell_emf(pmfmhd_ctx* c, const pmfmhd_grid* g, float* const U[9], float* ct,
                                           float dt, void* stream) {
  if (c == nullptr || U == nullptr || ct == nullptr) return PMFMHD_EINVAL;
  int rc = check_grid(g);
  if (rc) return rc;
  Cube G;
  if ((rc = cube_of(g, &G))) return rc;
  for (int f = 4; f < 9; ++f)
    if (!U[f]) return PMFMHD_EINVAL;
  if (!std::isfinite(dt)) return PMFMHD_EINVAL;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const long long n = ncells(g);
  const int nb = aux_blocks(c, n);
  auto slot = [&](int q) { return ct + (size_t)q * n; };
  edge_kernel<<<nb, kT, 0, s>>>(slot(CT_ECX), slot(CT_ECY), slot(CT_ECZ), slot(CT_EX), slot(CT_EY), slot(CT_EZ), G);
  face_euler_kernel<<<nb, kT, 0, s>>>(slot(CT_BXF), slot(CT_BYF), slot(CT_BZF), slot(CT_RBX), slot(CT_RBY),
                                      slot(CT_RBZ), slot(CT_EX), slot(CT_EY), slot(CT_EZ), G, dt, 1.0f / g->dx);
  face_average_kernel<<<nb, kT, 0, s>>>(slot(CT_BXF), slot(CT_BYF), slot(CT_BZF), U[5], U[6], U[7], U[4], U[8], G, 2);
  PMF_CK(cudaGetLastError());
  return PMFMHD_OK;
}

}  // extern "C"
