// Memory-bound companion kernels of the step: signal-speed reduction, FP64 diagnostics,
// the constrained-transport EMF / face / cell-B update, CT initialisation from a vector
// potential, and the device-side CFL timestep for the batched driver.
#pragma once
#include "physics.cuh"

namespace pmf {

constexpr int AUX_THREADS = 256;

// Nine field pointers passed by value.
struct CPtr9 { const float* p[9]; };
struct MPtr9 { float* p[9]; };

// Periodic neighbour index in one direction (CT is periodic-only, ct.jl:33-35).
__device__ __forceinline__ int wrap_inc(int i, int n) { return i + 1 == n ? 0 : i + 1; }
__device__ __forceinline__ int wrap_dec(int i, int n) { return i == 0 ? n - 1 : i - 1; }

template <class T> __device__ __forceinline__ T block_reduce_max(T v) {
  __shared__ T red[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  v = (threadIdx.x < (blockDim.x >> 5)) ? red[lane] : T(0);
  if (w == 0) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  }
  return v;
}

// max over cells of max_d(|v_d| + c_f,d)  (timestep.jl:4-14), one atomic per block
static __global__ void __launch_bounds__(AUX_THREADS) wavespeed_kernel(const CPtr9 U, int nc, Phys P,
                                                                unsigned int* out_bits) {
  float m = 0.0f;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
    F9 u;
#pragma unroll
    for (int f = 0; f < 9; ++f) u[f] = __ldg(U.p[f] + c);
    m = fmaxf(m, cell_wavespeed(u, P));
  }
  m = block_reduce_max(m);
  if (threadIdx.x == 0) atomicMax(out_bits, __float_as_uint(m));
}

// max |div B| by BC-aware centred differences, in FP64 (diagnostics.jl:6-20)
static __global__ void __launch_bounds__(AUX_THREADS) divb_kernel(const float* __restrict__ bx, const float* __restrict__ by,
                                                           const float* __restrict__ bz, int nx, int ny, int nz,
                                                           int bcx, int bcy, int bcz, double inv2dx,
                                                           unsigned long long* out_bits) {
  const int nc = nx * ny * nz;
  double m = 0.0;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
    const int i = c % nx, j = (c / nx) % ny, k = c / (nx * ny);
    float fxp, fxm, fyp, fym, fzp, fzm;
    const int ip = bc_index(i + 1, nx, bcx, &fxp), im = bc_index(i - 1, nx, bcx, &fxm);
    const int jp = bc_index(j + 1, ny, bcy, &fyp), jm = bc_index(j - 1, ny, bcy, &fym);
    const int kp = bc_index(k + 1, nz, bcz, &fzp), km = bc_index(k - 1, nz, bcz, &fzm);
    auto L = [&](int a, int b, int d) { return (d * ny + b) * nx + a; };
    const double db = ((double)bx[L(ip, j, k)] * fxp - (double)bx[L(im, j, k)] * fxm +
                       (double)by[L(i, jp, k)] * fyp - (double)by[L(i, jm, k)] * fym +
                       (double)bz[L(i, j, kp)] * fzp - (double)bz[L(i, j, km)] * fzm) * inv2dx;
    m = fmax(m, fabs(db));
  }
  m = block_reduce_max(m);
  if (threadIdx.x == 0) atomicMax(out_bits, (unsigned long long)__double_as_longlong(m));
}

// max face divergence of a CT face field, FP64 (ct.jl:176-185)
static __global__ void __launch_bounds__(AUX_THREADS) divb_face_kernel(const float* __restrict__ bxf,
                                                                const float* __restrict__ byf,
                                                                const float* __restrict__ bzf, int nx, int ny,
                                                                int nz, double invdx,
                                                                unsigned long long* out_bits) {
  const int nc = nx * ny * nz;
  double m = 0.0;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
    const int i = c % nx, j = (c / nx) % ny, k = c / (nx * ny);
    const int nxy = nx * ny;
    const double d = (((double)bxf[k * nxy + j * nx + wrap_inc(i, nx)] - bxf[c]) +
                      ((double)byf[k * nxy + wrap_inc(j, ny) * nx + i] - byf[c]) +
                      ((double)bzf[wrap_inc(k, nz) * nxy + j * nx + i] - bzf[c])) * invdx;
    m = fmax(m, fabs(d));
  }
  m = block_reduce_max(m);
  if (threadIdx.x == 0) atomicMax(out_bits, (unsigned long long)__double_as_longlong(m));
}

// Deterministic FP64 field sums: per-block partials (fixed order), then one block folds them.
static __global__ void __launch_bounds__(AUX_THREADS) totals_partial_kernel(const CPtr9 U, int nc,
                                                                     double* partial) {
  __shared__ double red[AUX_THREADS / 32][8];
  double s[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) s[q] = 0.0;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
#pragma unroll
    for (int q = 0; q < 8; ++q) s[q] += (double)__ldg(U.p[q] + c);
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 8; ++q) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s[q] += __shfl_down_sync(0xffffffffu, s[q], o);
    if (lane == 0) red[w][q] = s[q];
  }
  __syncthreads();
  if (threadIdx.x < 8) {
    double t = 0.0;
    for (int i = 0; i < AUX_THREADS / 32; ++i) t += red[i][threadIdx.x];
    partial[blockIdx.x * 8 + threadIdx.x] = t;
  }
}
static __global__ void totals_final_kernel(const double* partial, int nblocks, double scale, double* out) {
  if (threadIdx.x < 8) {
    double t = 0.0;
    for (int b = 0; b < nblocks; ++b) t += partial[b * 8 + threadIdx.x];
    out[threadIdx.x] = t * scale;
  }
}

// ---- constrained transport (ct.jl:57-143) ------------------------------------------------
// Gardiner & Stone 2005 contact-upwinded edge EMF (ct.jl:57-66)
__device__ __forceinline__ float gs05(float Ea0, float Eam, float Eb0, float Ebm, float mA0, float mAm, float mB0,
                                      float mBm, float Er00, float Erm0, float Er0m, float Ermm) {
  auto up = [](float m, float lower, float upper) {
    return m > 0.0f ? lower : (m < 0.0f ? upper : 0.5f * (lower + upper));
  };
  const float A1 = up(mA0, Erm0 - Ebm, Er00 - Eb0);
  const float A3 = up(mAm, Ebm - Ermm, Eb0 - Er0m);
  const float B1 = up(mB0, Er0m - Eam, Er00 - Ea0);
  const float B3 = up(mBm, Eam - Ermm, Ea0 - Erm0);
  return 0.25f * (((Ea0 + Eam + Eb0 + Ebm) + (A3 - A1)) + (B3 - B1));
}

// CTState slot layout (state.jl:44-52): slot s of cell c at packed[s*nc + c].
enum { CT_BXF = 0, CT_BYF, CT_BZF, CT_MFX, CT_MFY, CT_MFZ, CT_FXBY, CT_FXBZ, CT_FYBX, CT_FYBZ, CT_FZBX, CT_FZBY,
       CT_ECX, CT_ECY, CT_ECZ, CT_EX, CT_EY, CT_EZ, CT_RBX, CT_RBY, CT_RBZ, CT_NSLOT };

// edge EMFs of cell c from the lower-face fluxes and cell EMFs (ct.jl:71-93). The inputs are
// read through the same buffer the EMFs are stored into, so all 36 loads are issued before the
// first store: the compiler may not move a load above a store that could alias it, and three
// load-compute-store rounds would cost three memory latencies per cell.
__device__ __forceinline__ void ct_emf_cell(float* __restrict__ ct, int nx, int ny, int nz, int c) {
  const int nxy = nx * ny, nc = nxy * nz;
  const float* W = ct;
  const int i = c % nx, j = (c / nx) % ny, k = c / nxy;
  const int im = wrap_dec(i, nx), jm = wrap_dec(j, ny), km = wrap_dec(k, nz);
  const int cim = k * nxy + j * nx + im, cjm = k * nxy + jm * nx + i, ckm = km * nxy + j * nx + i;
  const int cimjm = k * nxy + jm * nx + im, cjmkm = km * nxy + jm * nx + i, ckmim = km * nxy + j * nx + im;
  auto w = [&](int s, int x) { return __ldg(W + (size_t)s * nc + x); };
  // z edge
  const float z0 = -w(CT_FXBY, c), z1 = -w(CT_FXBY, cjm), z2 = w(CT_FYBX, c), z3 = w(CT_FYBX, cim);
  const float z4 = w(CT_MFX, c), z5 = w(CT_MFX, cjm), z6 = w(CT_MFY, c), z7 = w(CT_MFY, cim);
  const float z8 = w(CT_ECZ, c), z9 = w(CT_ECZ, cim), z10 = w(CT_ECZ, cjm), z11 = w(CT_ECZ, cimjm);
  // x edge
  const float x0 = -w(CT_FYBZ, c), x1 = -w(CT_FYBZ, ckm), x2 = w(CT_FZBY, c), x3 = w(CT_FZBY, cjm);
  const float x4 = w(CT_MFY, ckm), x5 = w(CT_MFZ, c), x6 = w(CT_MFZ, cjm);
  const float x7 = w(CT_ECX, c), x8 = w(CT_ECX, cjm), x9 = w(CT_ECX, ckm), x10 = w(CT_ECX, cjmkm);
  // y edge
  const float y0 = -w(CT_FZBX, c), y1 = -w(CT_FZBX, cim), y2 = w(CT_FXBZ, c), y3 = w(CT_FXBZ, ckm);
  const float y4 = w(CT_MFZ, cim), y5 = w(CT_MFX, ckm);
  const float y6 = w(CT_ECY, c), y7 = w(CT_ECY, ckm), y8 = w(CT_ECY, cim), y9 = w(CT_ECY, ckmim);
  const float ez = gs05(z0, z1, z2, z3, z4, z5, z6, z7, z8, z9, z10, z11);
  const float ex = gs05(x0, x1, x2, x3, z6, x4, x5, x6, x7, x8, x9, x10);
  const float ey = gs05(y0, y1, y2, y3, x5, y4, z4, y5, y6, y7, y8, y9);
  ct[(size_t)CT_EZ * nc + c] = ez;
  ct[(size_t)CT_EX * nc + c] = ex;
  ct[(size_t)CT_EY * nc + c] = ey;
}

static __global__ void __launch_bounds__(AUX_THREADS) ct_emf_kernel(float* __restrict__ ct, int nx, int ny, int nz) {
  const int nc = nx * ny * nz;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) ct_emf_cell(ct, nx, ny, nz, c);
}

// face update of cell c by the discrete curl of the edge EMFs, plain or Kahan (ct.jl:96-129)
template <bool COMP>
__device__ __forceinline__ void ct_face_cell(float* __restrict__ ct, int nx, int ny, int nz, float dtdx, int c) {
  const int nxy = nx * ny, nc = nxy * nz;
  const float* ex = ct + (size_t)CT_EX * nc;
  const float* ey = ct + (size_t)CT_EY * nc;
  const float* ez = ct + (size_t)CT_EZ * nc;
  const int i = c % nx, j = (c / nx) % ny, k = c / nxy;
  const int ip = k * nxy + j * nx + wrap_inc(i, nx), jp = k * nxy + wrap_inc(j, ny) * nx + i,
            kp = wrap_inc(k, nz) * nxy + j * nx + i;
  const float dbx = dtdx * ((ez[jp] - ez[c]) - (ey[kp] - ey[c]));
  const float dby = dtdx * ((ex[kp] - ex[c]) - (ez[ip] - ez[c]));
  const float dbz = dtdx * ((ey[ip] - ey[c]) - (ex[jp] - ex[c]));
  float* bxf = ct + (size_t)CT_BXF * nc;
  float* byf = ct + (size_t)CT_BYF * nc;
  float* bzf = ct + (size_t)CT_BZF * nc;
  // every load before the first store (the faces, remainders and EMFs share one buffer)
  const float fx = bxf[c], fy = byf[c], fz = bzf[c];
  if (COMP) {
    float* rbx = ct + (size_t)CT_RBX * nc;
    float* rby = ct + (size_t)CT_RBY * nc;
    float* rbz = ct + (size_t)CT_RBZ * nc;
    float rx = rbx[c], ry = rby[c], rz = rbz[c];
    const float nbx = comp_add(fx, -dbx, rx), nby = comp_add(fy, -dby, ry), nbz = comp_add(fz, -dbz, rz);
    bxf[c] = nbx;
    byf[c] = nby;
    bzf[c] = nbz;
    rbx[c] = rx;
    rby[c] = ry;
    rbz[c] = rz;
  } else {
    bxf[c] = fx - dbx;
    byf[c] = fy - dby;
    bzf[c] = fz - dbz;
  }
}

template <bool COMP>
static __global__ void __launch_bounds__(AUX_THREADS) ct_face_kernel(float* __restrict__ ct, int nx, int ny, int nz,
                                                              float dtdx) {
  const int nc = nx * ny * nz;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x)
    ct_face_cell<COMP>(ct, nx, ny, nz, dtdx, c);
}

// cell B of cell c = face average (ct.jl:132-143); returns the new state's signal speed
__device__ __forceinline__ float ct_bcc_cell(const float* __restrict__ ct, const MPtr9& Un, int nx, int ny, int nz,
                                             const Phys& P, bool want_speed, int c) {
  const int nxy = nx * ny, nc = nxy * nz;
  const float* bxf = ct + (size_t)CT_BXF * nc;
  const float* byf = ct + (size_t)CT_BYF * nc;
  const float* bzf = ct + (size_t)CT_BZF * nc;
  const int i = c % nx, j = (c / nx) % ny, k = c / nxy;
  const float bx = 0.5f * (bxf[c] + bxf[k * nxy + j * nx + wrap_inc(i, nx)]);
  const float by = 0.5f * (byf[c] + byf[k * nxy + wrap_inc(j, ny) * nx + i]);
  const float bz = 0.5f * (bzf[c] + bzf[wrap_inc(k, nz) * nxy + j * nx + i]);
  // the hydro fields are read before the B stores (all nine fields may share one buffer)
  F9 u{{0.0f, 0.0f, 0.0f, 0.0f, 0.0f, bx, by, bz, 0.0f}};
  if (want_speed)
    for (int f = 0; f < 5; ++f) u[f] = Un.p[f][c];
  Un.p[5][c] = bx;
  Un.p[6][c] = by;
  Un.p[7][c] = bz;
  if (!want_speed) return 0.0f;
  return cell_wavespeed(u, P);
}

static __global__ void __launch_bounds__(AUX_THREADS) ct_bcc_kernel(const float* __restrict__ ct, const MPtr9 Un, int nx,
                                                             int ny, int nz, Phys P, unsigned int* smax_bits) {
  const int nc = nx * ny * nz;
  float m = 0.0f;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x)
    m = fmaxf(m, ct_bcc_cell(ct, Un, nx, ny, nz, P, smax_bits != nullptr, c));
  if (smax_bits != nullptr) {
    m = block_reduce_max(m);
    if (threadIdx.x == 0) atomicMax(smax_bits, __float_as_uint(m));
  }
}

// faces = discrete curl of an edge potential (ct.jl:310-320)
static __global__ void __launch_bounds__(AUX_THREADS) ct_curl_kernel(const float* __restrict__ Ax,
                                                              const float* __restrict__ Ay,
                                                              const float* __restrict__ Az, float* __restrict__ ct,
                                                              int nx, int ny, int nz, float invdx) {
  const int nxy = nx * ny, nc = nxy * nz;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
    const int i = c % nx, j = (c / nx) % ny, k = c / nxy;
    const int ip = k * nxy + j * nx + wrap_inc(i, nx), jp = k * nxy + wrap_inc(j, ny) * nx + i,
              kp = wrap_inc(k, nz) * nxy + j * nx + i;
    ct[(size_t)CT_BXF * nc + c] = ((Az[jp] - Az[c]) - (Ay[kp] - Ay[c])) * invdx;
    ct[(size_t)CT_BYF * nc + c] = ((Ax[kp] - Ax[c]) - (Az[ip] - Az[c])) * invdx;
    ct[(size_t)CT_BZF * nc + c] = ((Ay[ip] - Ay[c]) - (Ax[jp] - Ax[c])) * invdx;
    ct[(size_t)CT_RBX * nc + c] = 0.0f;
    ct[(size_t)CT_RBY * nc + c] = 0.0f;
    ct[(size_t)CT_RBZ * nc + c] = 0.0f;
  }
}

// cell B <- face average, E keeps the thermal pressure, psi <- 0 (ct.jl:205-219)
static __global__ void __launch_bounds__(AUX_THREADS) ct_cell_from_faces_kernel(const float* __restrict__ ct,
                                                                         const MPtr9 U, int nx, int ny, int nz) {
  const int nxy = nx * ny, nc = nxy * nz;
  const float* bxf = ct + (size_t)CT_BXF * nc;
  const float* byf = ct + (size_t)CT_BYF * nc;
  const float* bzf = ct + (size_t)CT_BZF * nc;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
    const int i = c % nx, j = (c / nx) % ny, k = c / nxy;
    const float bx = 0.5f * (bxf[c] + bxf[k * nxy + j * nx + wrap_inc(i, nx)]);
    const float by = 0.5f * (byf[c] + byf[k * nxy + wrap_inc(j, ny) * nx + i]);
    const float bz = 0.5f * (bzf[c] + bzf[wrap_inc(k, nz) * nxy + j * nx + i]);
    const float ox = U.p[5][c], oy = U.p[6][c], oz = U.p[7][c];
    U.p[4][c] += 0.5f * ((bx * bx + by * by + bz * bz) - (ox * ox + oy * oy + oz * oz));
    U.p[5][c] = bx;
    U.p[6][c] = by;
    U.p[7][c] = bz;
    U.p[8][c] = 0.0f;
  }
}

}  // namespace pmf
