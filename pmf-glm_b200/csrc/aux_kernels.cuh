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

// ---- CT companion kernels: column forms -------------------------------------------------
// One thread per (x, y) column of a 32 x 8 tile marches a chunk of CTC_Z planes in z: the
// cell index needs no division, every slot has its own restrict pointer (so the compiler
// may overlap one plane's loads with the last plane's stores), and the values of plane k
// that plane k+1 reads again as its lower neighbour stay in registers (25 loads per cell
// for the EMFs, of the 36 values its stencil touches). Per cell: the Gardiner & Stone EMFs (ct.jl:71-93), the face
// update (ct.jl:96-129) and the face-average cell B (ct.jl:132-143).
constexpr int CTC_X = 32, CTC_Y = AUX_THREADS / 32, CTC_Z = 16;
inline dim3 ctc_grid(int nx, int ny, int nz) {
  return dim3((nx + CTC_X - 1) / CTC_X, (ny + CTC_Y - 1) / CTC_Y, (nz + CTC_Z - 1) / CTC_Z);
}

// The column bodies: tile (tx, ty), z chunk tz; thread t of AUX_THREADS owns column
// (tx*32 + t%32, ty*CTC_Y + t/32). Used by the single-box kernels below and by the batched
// driver, which maps its blocks to (box, tile).

// edge EMFs (ct.jl:71-93)
__device__ __forceinline__ void ct_emf_col(
    const float* __restrict__ MFX, const float* __restrict__ MFY, const float* __restrict__ MFZ,
    const float* __restrict__ FXBY, const float* __restrict__ FXBZ, const float* __restrict__ FYBX,
    const float* __restrict__ FYBZ, const float* __restrict__ FZBX, const float* __restrict__ FZBY,
    const float* __restrict__ ECX, const float* __restrict__ ECY, const float* __restrict__ ECZ,
    float* __restrict__ EX, float* __restrict__ EY, float* __restrict__ EZ, int nx, int ny, int nz, int tx, int ty,
    int tz) {
  const int i = tx * CTC_X + (threadIdx.x & 31), j = ty * CTC_Y + (threadIdx.x >> 5);
  if (i >= nx || j >= ny) return;
  const int z0 = tz * CTC_Z, z1 = min(z0 + CTC_Z, nz);
  const size_t nxy = (size_t)nx * ny;
  const int im = wrap_dec(i, nx), jm = wrap_dec(j, ny);
  const size_t o = (size_t)j * nx + i, oim = (size_t)j * nx + im, ojm = (size_t)jm * nx + i,
               oimjm = (size_t)jm * nx + im;
  // plane k-1 values of the x and y edges
  size_t b = (size_t)wrap_dec(z0, nz) * nxy;
  float pFYBZ = FYBZ[b + o], pMFY = MFY[b + o], pECX = ECX[b + o], pECXjm = ECX[b + ojm];
  float pFXBZ = FXBZ[b + o], pMFX = MFX[b + o], pECY = ECY[b + o], pECYim = ECY[b + oim];
  for (int k = z0; k < z1; ++k) {
    b = (size_t)k * nxy;
    const float fxby = FXBY[b + o], fxby_jm = FXBY[b + ojm], fybx = FYBX[b + o], fybx_im = FYBX[b + oim];
    const float mfx = MFX[b + o], mfx_jm = MFX[b + ojm], mfy = MFY[b + o], mfy_im = MFY[b + oim];
    const float ecz = ECZ[b + o], ecz_im = ECZ[b + oim], ecz_jm = ECZ[b + ojm], ecz_imjm = ECZ[b + oimjm];
    const float fybz = FYBZ[b + o], fzby = FZBY[b + o], fzby_jm = FZBY[b + ojm], mfz = MFZ[b + o];
    const float mfz_jm = MFZ[b + ojm], ecx = ECX[b + o], ecx_jm = ECX[b + ojm];
    const float fzbx = FZBX[b + o], fzbx_im = FZBX[b + oim], fxbz = FXBZ[b + o], mfz_im = MFZ[b + oim];
    const float ecy = ECY[b + o], ecy_im = ECY[b + oim];
    EZ[b + o] = gs05(-fxby, -fxby_jm, fybx, fybx_im, mfx, mfx_jm, mfy, mfy_im, ecz, ecz_im, ecz_jm, ecz_imjm);
    EX[b + o] = gs05(-fybz, -pFYBZ, fzby, fzby_jm, mfy, pMFY, mfz, mfz_jm, ecx, ecx_jm, pECX, pECXjm);
    EY[b + o] = gs05(-fzbx, -fzbx_im, fxbz, pFXBZ, mfz, mfz_im, mfx, pMFX, ecy, pECY, ecy_im, pECYim);
    pFYBZ = fybz; pMFY = mfy; pECX = ecx; pECXjm = ecx_jm;
    pFXBZ = fxbz; pMFX = mfx; pECY = ecy; pECYim = ecy_im;
  }
}

// face update by the discrete curl of the edge EMFs, plain or Kahan (ct.jl:96-129)
template <bool COMP>
__device__ __forceinline__ void ct_face_col(const float* __restrict__ ex, const float* __restrict__ ey,
                                            const float* __restrict__ ez, float* __restrict__ bxf,
                                            float* __restrict__ byf, float* __restrict__ bzf, float* __restrict__ rbx,
                                            float* __restrict__ rby, float* __restrict__ rbz, int nx, int ny, int nz,
                                            float dtdx, int tx, int ty, int tz) {
  const int i = tx * CTC_X + (threadIdx.x & 31), j = ty * CTC_Y + (threadIdx.x >> 5);
  if (i >= nx || j >= ny) return;
  const int z0 = tz * CTC_Z, z1 = min(z0 + CTC_Z, nz);
  const size_t nxy = (size_t)nx * ny;
  const size_t o = (size_t)j * nx + i, oip = (size_t)j * nx + wrap_inc(i, nx), ojp = (size_t)wrap_inc(j, ny) * nx + i;
  // plane k values that plane k-1 read as its upper neighbour
  float ex_c = ex[(size_t)z0 * nxy + o], ey_c = ey[(size_t)z0 * nxy + o];
  for (int k = z0; k < z1; ++k) {
    const size_t b = (size_t)k * nxy, bp = (size_t)wrap_inc(k, nz) * nxy;
    const float ez_c = ez[b + o], ez_jp = ez[b + ojp], ez_ip = ez[b + oip], ey_ip = ey[b + oip], ex_jp = ex[b + ojp];
    const float ey_kp = ey[bp + o], ex_kp = ex[bp + o];
    const float dbx = dtdx * ((ez_jp - ez_c) - (ey_kp - ey_c));
    const float dby = dtdx * ((ex_kp - ex_c) - (ez_ip - ez_c));
    const float dbz = dtdx * ((ey_ip - ey_c) - (ex_jp - ex_c));
    const float fx = bxf[b + o], fy = byf[b + o], fz = bzf[b + o];
    if (COMP) {
      float rx = rbx[b + o], ry = rby[b + o], rz = rbz[b + o];
      const float nbx = comp_add(fx, -dbx, rx), nby = comp_add(fy, -dby, ry), nbz = comp_add(fz, -dbz, rz);
      bxf[b + o] = nbx;
      byf[b + o] = nby;
      bzf[b + o] = nbz;
      rbx[b + o] = rx;
      rby[b + o] = ry;
      rbz[b + o] = rz;
    } else {
      bxf[b + o] = fx - dbx;
      byf[b + o] = fy - dby;
      bzf[b + o] = fz - dbz;
    }
    ex_c = ex_kp;
    ey_c = ey_kp;
  }
}

// cell B = face average (ct.jl:132-143); returns this thread's max signal speed of the new
// state (0 without want_speed). Every thread returns: the caller reduces over the block.
__device__ __forceinline__ float ct_bcc_col(const float* __restrict__ bxf, const float* __restrict__ byf,
                                            const float* __restrict__ bzf, const MPtr9& Un, int nx, int ny, int nz,
                                            const Phys& P, bool want_speed, int tx, int ty, int tz) {
  const int i = tx * CTC_X + (threadIdx.x & 31), j = ty * CTC_Y + (threadIdx.x >> 5);
  float m = 0.0f;
  if (i >= nx || j >= ny) return m;
  const int z0 = tz * CTC_Z, z1 = min(z0 + CTC_Z, nz);
  const size_t nxy = (size_t)nx * ny;
  const size_t o = (size_t)j * nx + i, oip = (size_t)j * nx + wrap_inc(i, nx), ojp = (size_t)wrap_inc(j, ny) * nx + i;
  float bz_c = bzf[(size_t)z0 * nxy + o];
  for (int k = z0; k < z1; ++k) {
    const size_t b = (size_t)k * nxy, c = b + o;
    const float bz_kp = bzf[(size_t)wrap_inc(k, nz) * nxy + o];
    const float bx = 0.5f * (bxf[c] + bxf[b + oip]);
    const float by = 0.5f * (byf[c] + byf[b + ojp]);
    const float bz = 0.5f * (bz_c + bz_kp);
    F9 u{{0.0f, 0.0f, 0.0f, 0.0f, 0.0f, bx, by, bz, 0.0f}};
    if (want_speed)
      for (int f = 0; f < 5; ++f) u[f] = Un.p[f][c];
    Un.p[5][c] = bx;
    Un.p[6][c] = by;
    Un.p[7][c] = bz;
    if (want_speed) m = fmaxf(m, cell_wavespeed(u, P));
    bz_c = bz_kp;
  }
  return m;
}

static __global__ void __launch_bounds__(AUX_THREADS) ct_emf_col_kernel(
    const float* __restrict__ MFX, const float* __restrict__ MFY, const float* __restrict__ MFZ,
    const float* __restrict__ FXBY, const float* __restrict__ FXBZ, const float* __restrict__ FYBX,
    const float* __restrict__ FYBZ, const float* __restrict__ FZBX, const float* __restrict__ FZBY,
    const float* __restrict__ ECX, const float* __restrict__ ECY, const float* __restrict__ ECZ,
    float* __restrict__ EX, float* __restrict__ EY, float* __restrict__ EZ, int nx, int ny, int nz) {
  ct_emf_col(MFX, MFY, MFZ, FXBY, FXBZ, FYBX, FYBZ, FZBX, FZBY, ECX, ECY, ECZ, EX, EY, EZ, nx, ny, nz, blockIdx.x,
             blockIdx.y, blockIdx.z);
}

template <bool COMP>
static __global__ void __launch_bounds__(AUX_THREADS) ct_face_col_kernel(
    const float* __restrict__ ex, const float* __restrict__ ey, const float* __restrict__ ez,
    float* __restrict__ bxf, float* __restrict__ byf, float* __restrict__ bzf, float* __restrict__ rbx,
    float* __restrict__ rby, float* __restrict__ rbz, int nx, int ny, int nz, float dtdx) {
  ct_face_col<COMP>(ex, ey, ez, bxf, byf, bzf, rbx, rby, rbz, nx, ny, nz, dtdx, blockIdx.x, blockIdx.y, blockIdx.z);
}

static __global__ void __launch_bounds__(AUX_THREADS) ct_bcc_col_kernel(
    const float* __restrict__ bxf, const float* __restrict__ byf, const float* __restrict__ bzf, const MPtr9 Un,
    int nx, int ny, int nz, Phys P, unsigned int* smax_bits) {
  float m = ct_bcc_col(bxf, byf, bzf, Un, nx, ny, nz, P, smax_bits != nullptr, blockIdx.x, blockIdx.y, blockIdx.z);
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
