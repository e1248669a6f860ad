// Initial conditions on the device: the Batchelor primordial-magnetic-field generator and
// the CT face construction from a cell field (both host FFTW code in the reference).
//
//   pmfmhd_pmf_batchelor_field  <- pmf_batchelor_field (lib/MHDKernels/src/pmf.jl:300-591)
//                                  with the physical-hash realizations (pmf.jl:109-191)
//   pmfmhd_pmf_install          <- _install_pmf_field! (pmf.jl:239-261), uniform gas part
//   pmfmhd_ct_faces_from_cells  <- ct_faces_from_cells! (ct.jl:246-308)
//
// The spectral coefficients are built by one kernel over the half-spectrum modes (counter-
// based hashed normals, so any mode can be generated independently of the others), the
// inverse transforms are cuFFT C2R / Z2D, and the reductions are FP64 in a fixed order.
// Rounding follows the reference where it matters for which modes are kept: wavenumbers,
// |k|^2 and the cutoff tests use the reference's operation order with explicitly rounded
// operations (no multiply-add contraction), as do the single-precision complex products.
#include <cufft.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <string>
#include <vector>

#include "host_internal.h"

namespace pmf {
namespace {

constexpr int kThreads = 256;

// ---- counter-based normal deviates keyed by physical mode (pmf.jl:109-141) ----------------
// SplitMix64's output function applied after a golden-ratio increment.
__device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
  unsigned long long z = x + 0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

__device__ __forceinline__ double hash_uniform(long long seed, long long qx, long long qy, long long qz, int comp,
                                               int lane) {
  unsigned long long h = mix64((unsigned long long)seed);
  h = mix64(h ^ (unsigned long long)qx);
  h = mix64(h ^ (unsigned long long)qy);
  h = mix64(h ^ (unsigned long long)qz);
  h = mix64(h ^ (unsigned long long)(long long)comp);
  h = mix64(h ^ (unsigned long long)(long long)lane);
  return __dmul_rn(__dadd_rn((double)(h >> 11), 0.5), 0x1.0p-53);
}

__device__ __forceinline__ float2 hash_normal(long long seed, long long qx, long long qy, long long qz, int comp,
                                              bool real_only) {
  const double u1 = hash_uniform(seed, qx, qy, qz, comp, 1);
  const double u2 = hash_uniform(seed, qx, qy, qz, comp, 2);
  const double radius = sqrt(__dmul_rn(-2.0, log(u1)));
  if (real_only) return make_float2((float)__dmul_rn(radius, cospi(__dmul_rn(2.0, u2))), 0.0f);
  const double phase = __dmul_rn(2.0 * M_PI, u2);
  return make_float2((float)__dmul_rn(radius, cos(phase)), (float)__dmul_rn(radius, sin(phase)));
}

__device__ __forceinline__ int mode_of(int i, int n) { return i <= n / 2 ? i : i - n; }

// Vector-potential coefficients of half-spectrum index (ii, jj, kk) of an (ox, oy, oz) grid
// (_physical_hash_vector_potential_k, pmf.jl:149-191): on the x = 0 and x = Nyquist planes the
// mode of the pair (-my, -mz) that comes later in (j, k) order is the conjugate of the earlier
// one, and self-paired modes are real.
__device__ void hash_potential(long long seed, int qscale, bool zero_phase, int ox, int oy, int oz, int ii, int jj,
                               int kk, float2 A[3]) {
  const int oxh = ox / 2 + 1;
  const int mx = ii, my = mode_of(jj, oy), mz = mode_of(kk, oz);
  bool conj = false, real_only = false;
  int key_my = my, key_mz = mz;
  if (ii == 0 || ii == oxh - 1) {
    const int pj = ((-my) % oy + oy) % oy, pk = ((-mz) % oz + oz) % oz;
    if (pj < jj || (pj == jj && pk < kk)) {
      conj = true;
      key_my = mode_of(pj, oy);
      key_mz = mode_of(pk, oz);
    } else if (pj == jj && pk == kk) {
      real_only = true;
    }
  }
  const long long qx = (long long)qscale * mx, qy = (long long)qscale * key_my, qz = (long long)qscale * key_mz;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    float2 v = hash_normal(seed, qx, qy, qz, c + 1, zero_phase || real_only);
    if (conj) v.y = -v.y;
    A[c] = v;
  }
}

// A realization on a source grid zero-padded into the target spectrum
// (_rfft_zero_pad_complex, pmf.jl:205-224): returns false where the source has no mode.
struct Source {
  int ox, oy, oz;
  bool same;    // the source grid is the target grid
  float scale;  // Float32(Vtarget / Vsource)
};

__device__ bool source_potential(long long seed, int qscale, bool zero_phase, const Source& S, int i, int j, int k,
                                 int mxt, int myt, int mzt, float2 A[3]) {
  if (S.same) {
    hash_potential(seed, qscale, zero_phase, S.ox, S.oy, S.oz, i, j, k, A);
    return true;
  }
  if (mxt > S.ox / 2 || myt > S.oy / 2 || myt < -(S.oy - 1 - S.oy / 2) || mzt > S.oz / 2 ||
      mzt < -(S.oz - 1 - S.oz / 2))
    return false;
  const int sj = myt >= 0 ? myt : S.oy + myt, sk = mzt >= 0 ? mzt : S.oz + mzt;
  hash_potential(seed, qscale, zero_phase, S.ox, S.oy, S.oz, mxt, sj, sk, A);
#pragma unroll
  for (int c = 0; c < 3; ++c) A[c] = make_float2(__fmul_rn(S.scale, A[c].x), __fmul_rn(S.scale, A[c].y));
  return true;
}

struct PmfModes {
  int nx, ny, nz, nxh;
  long long seed;
  int qscale;
  bool zero_phase;
  double two_pi_over_L;
  double km2;        // kmax^2 (infinite: no band limit)
  double kmin2;      // kmin^2
  double kc, low_kc;
  double low_thr;    // Float32(preserve_low_kmax)^2 * (1 + 8 eps_f32), as a double; < 0: no low band
  double amp_exp, order, energy_index;
  float high_source_scale;
  int invariant_axis;
  bool fixed_power, project;
  Source high, low;
  const float* sym;  // sx[nxh] sy[ny] sz[nz] rx[nxh] ry[ny] rz[nz]
};

__device__ __forceinline__ float2 cmul_r(float s, float2 z) { return make_float2(__fmul_rn(s, z.x), __fmul_rn(s, z.y)); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y)); }
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y)); }
__device__ __forceinline__ float2 times_i(float2 z) { return make_float2(-z.y, z.x); }
__device__ __forceinline__ float abs2(float2 z) { return __fadd_rn(__fmul_rn(z.x, z.x), __fmul_rn(z.y, z.y)); }

// One half-spectrum mode of B = i r x (amp A) (pmf.jl:458-509), optionally projected onto the
// target grid's centred-difference solenoidal subspace, band-limited and rescaled to the
// analytic envelope (pmf.jl:520-556). bk: 3 field spectra; lk: the preserved low band or null.
__global__ void __launch_bounds__(kThreads) pmf_modes_kernel(const PmfModes P, float2* __restrict__ bk,
                                                             float2* __restrict__ lk) {
  const long long nck = (long long)P.nxh * P.ny * P.nz;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < nck;
       idx += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(idx % P.nxh);
    const int j = (int)((idx / P.nxh) % P.ny);
    const int k = (int)(idx / ((long long)P.nxh * P.ny));
    const int mx = i, my = mode_of(j, P.ny), mz = mode_of(k, P.nz);
    const double kx = __dmul_rn((double)mx, P.two_pi_over_L);
    const double ky = __dmul_rn((double)my, P.two_pi_over_L);
    const double kz = __dmul_rn((double)mz, P.two_pi_over_L);
    const double k2 = __dadd_rn(__dadd_rn(__dmul_rn(kx, kx), __dmul_rn(ky, ky)), __dmul_rn(kz, kz));
    float2 b[3] = {{0.f, 0.f}, {0.f, 0.f}, {0.f, 0.f}};
    bool use_low = false;
    const int inv_m = P.invariant_axis == 1 ? mx : (P.invariant_axis == 2 ? my : mz);
    if (!(k2 == 0.0 || k2 > P.km2 || (P.invariant_axis != 0 && inv_m != 0))) {
      const double kmag = sqrt(k2);
      use_low = P.low_thr >= 0.0 && k2 <= P.low_thr;
      const double lkc = use_low ? P.low_kc : P.kc;
      const double ratio = kmag / lkc;
      const double amp = __dmul_rn(pow(ratio, P.amp_exp), exp(__dmul_rn(-0.5, pow(ratio, P.order))));
      float2 A[3];
      const bool have = use_low ? source_potential(P.seed, P.qscale, P.zero_phase, P.low, i, j, k, mx, my, mz, A)
                                : source_potential(P.seed, P.qscale, P.zero_phase, P.high, i, j, k, mx, my, mz, A);
      if (have) {
        const float w = (float)__dmul_rn(amp, (double)(use_low ? 1.0f : P.high_source_scale));
        const float2 wa[3] = {cmul_r(w, A[0]), cmul_r(w, A[1]), cmul_r(w, A[2])};
        const float* sym = P.sym;
        const float sx = sym[i], sy = sym[P.nxh + j], sz = sym[P.nxh + P.ny + k];
        const int roff = P.nxh + P.ny + P.nz;
        const float rx = sym[roff + i], ry = sym[roff + P.nxh + j], rz = sym[roff + P.nxh + P.ny + k];
        b[0] = times_i(csub(cmul_r(ry, wa[2]), cmul_r(rz, wa[1])));
        b[1] = times_i(csub(cmul_r(rz, wa[0]), cmul_r(rx, wa[2])));
        b[2] = times_i(csub(cmul_r(rx, wa[1]), cmul_r(ry, wa[0])));
        if (P.project) {
          const float s2 = __fadd_rn(__fadd_rn(__fmul_rn(sx, sx), __fmul_rn(sy, sy)), __fmul_rn(sz, sz));
          if (s2 > 0.0f) {
            const float2 dot = cadd(cadd(cmul_r(sx, b[0]), cmul_r(sy, b[1])), cmul_r(sz, b[2]));
            const float2 par = make_float2(__fdiv_rn(dot.x, s2), __fdiv_rn(dot.y, s2));
            b[0] = csub(b[0], cmul_r(sx, par));
            b[1] = csub(b[1], cmul_r(sy, par));
            b[2] = csub(b[2], cmul_r(sz, par));
          }
        }
      }
    }
    float2 lo[3] = {use_low ? b[0] : make_float2(0.f, 0.f), use_low ? b[1] : make_float2(0.f, 0.f),
                    use_low ? b[2] : make_float2(0.f, 0.f)};
    const bool below_kmin = P.kmin2 > 0.0 && k2 <= P.kmin2;
    if (below_kmin) b[0] = b[1] = b[2] = make_float2(0.f, 0.f);
    if (P.fixed_power && !(k2 == 0.0 || k2 > P.km2 || k2 <= P.kmin2)) {
      const float raw = __fadd_rn(__fadd_rn(abs2(b[0]), abs2(b[1])), abs2(b[2]));
      if (raw > 0.0f) {
        const double kmag = sqrt(k2);
        const double lkc = use_low ? P.low_kc : P.kc;
        const double ratio = kmag / lkc;
        const double target = __dmul_rn(pow(ratio, P.energy_index - 2.0), exp(-pow(ratio, P.order)));
        const float sm = (float)sqrt(target / (double)raw);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          b[c] = cmul_r(sm, b[c]);
          if (use_low) lo[c] = cmul_r(sm, lo[c]);
        }
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      bk[c * nck + idx] = b[c];
      if (lk) lk[c * nck + idx] = lo[c];
    }
  }
}

// x <- x * mul (when `write`), partial[b] = sum of (x * mul)^2 over block b's cells (FP64)
__global__ void __launch_bounds__(kThreads) scale_sumsq_kernel(const float* src, float* x, long long n, float mul,
                                                               bool write, double* __restrict__ partial) {
  __shared__ double red[kThreads / 32];
  double acc = 0.0;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    const float v = src[c] * mul;
    if (write) x[c] = v;
    acc += (double)v * (double)v;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) t += red[w];
    partial[blockIdx.x] = t;
  }
}

// out[slot] = sum of partial[0..nb) in block order
__global__ void fold_kernel(const double* __restrict__ partial, int nb, double* __restrict__ out, int slot) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    double t = 0.0;
    for (int b = 0; b < nb; ++b) t += partial[b];
    out[slot] = t;
  }
}

// Uniform gas around an installed field (pmf.jl:239-261): rho, zero momentum,
// E = p0/(gamma-1) + |B|^2/2, psi = 0.
__global__ void __launch_bounds__(kThreads) pmf_install_kernel(float* __restrict__ rho, float* __restrict__ mx,
                                                               float* __restrict__ my, float* __restrict__ mz,
                                                               float* __restrict__ E, const float* __restrict__ bx,
                                                               const float* __restrict__ by,
                                                               const float* __restrict__ bz, float* __restrict__ psi,
                                                               long long n, float rho0, float eth) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    const float b1 = bx[c], b2 = by[c], b3 = bz[c];
    rho[c] = rho0;
    mx[c] = 0.0f;
    my[c] = 0.0f;
    mz[c] = 0.0f;
    E[c] = eth + 0.5f * (b1 * b1 + b2 * b2 + b3 * b3);
    psi[c] = 0.0f;
  }
}

// Periodic repetition of a tile (_periodic_tile_field, pmf.jl:226-237)
__global__ void __launch_bounds__(kThreads) tile_kernel(const float* __restrict__ src, int sx, int sy, int sz,
                                                        float* __restrict__ dst, int nx, int ny, long long n) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / ((long long)nx * ny));
    dst[c] = src[((long long)(k % sz) * sy + (j % sy)) * sx + (i % sx)];
  }
}

// ---- ct_faces_from_cells! (ct.jl:246-308), FP64 like the reference's host code ------------
__global__ void __launch_bounds__(kThreads) to_double_kernel(const float* __restrict__ a, double* __restrict__ d,
                                                             long long n) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x)
    d[c] = (double)a[c];
}

// Half-cell phase of index m on an n-point axis and whether it is the Nyquist index
// (_ct_half_phase, ct.jl:240-244).
__device__ __forceinline__ double half_phase(int m, int n, bool* nyq) {
  *nyq = (n % 2 == 0) && m == n / 2;
  const int mm = (double)m > n / 2.0 ? m - n : m;
  return *nyq ? 0.0 : M_PI * mm / n;
}

// Project each mode onto t.b = 0 (t = tan(theta)) and build the face spectra
// f_d = b_d exp(-i theta_d) / cos(theta_d); Nyquist components are dropped (ct.jl:278-297).
__global__ void __launch_bounds__(kThreads) ct_face_modes_kernel(double2* __restrict__ bh, int nx, int ny, int nz) {
  const int nxh = nx / 2 + 1;
  const long long nck = (long long)nxh * ny * nz;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < nck;
       idx += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(idx % nxh), j = (int)((idx / nxh) % ny), k = (int)(idx / ((long long)nxh * ny));
    bool qx, qy, qz;
    const double th[3] = {half_phase(i, nx, &qx), half_phase(j, ny, &qy), half_phase(k, nz, &qz)};
    const bool nyq[3] = {qx, qy, qz};
    double2 b[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) b[d] = nyq[d] ? make_double2(0.0, 0.0) : bh[d * nck + idx];
    const double t[3] = {tan(th[0]), tan(th[1]), tan(th[2])};
    const double t2 = t[0] * t[0] + t[1] * t[1] + t[2] * t[2];
    if (t2 > 0.0) {
      const double2 dot = make_double2((t[0] * b[0].x + t[1] * b[1].x + t[2] * b[2].x) / t2,
                                       (t[0] * b[0].y + t[1] * b[1].y + t[2] * b[2].y) / t2);
#pragma unroll
      for (int d = 0; d < 3; ++d) b[d] = make_double2(b[d].x - t[d] * dot.x, b[d].y - t[d] * dot.y);
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double c = cos(th[d]), s = sin(th[d]);
      // b * (cos - i sin) / cos
      bh[d * nck + idx] = make_double2((b[d].x * c + b[d].y * s) / c, (b[d].y * c - b[d].x * s) / c);
    }
  }
}

__global__ void __launch_bounds__(kThreads) faces_to_float_kernel(const double* __restrict__ f, float* __restrict__ out,
                                                                  long long n, double inv_n) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x)
    out[c] = (float)(f[c] * inv_n);
}

// partial sums of (new - old)^2, old^2 and new^2 of the three cell-B components
__global__ void __launch_bounds__(kThreads) ct_change_kernel(const float* __restrict__ b0, const float* __restrict__ b1,
                                                             const float* __restrict__ b2,
                                                             const double* __restrict__ o0,
                                                             const double* __restrict__ o1,
                                                             const double* __restrict__ o2, long long n,
                                                             double* __restrict__ partial) {
  __shared__ double red[3][kThreads / 32];
  double a[3] = {0.0, 0.0, 0.0};
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    const double nb[3] = {(double)b0[c], (double)b1[c], (double)b2[c]};
    const double ob[3] = {o0[c], o1[c], o2[c]};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      a[0] += (nb[d] - ob[d]) * (nb[d] - ob[d]);
      a[1] += ob[d] * ob[d];
      a[2] += nb[d] * nb[d];
    }
  }
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    for (int o = 16; o > 0; o >>= 1) a[q] += __shfl_down_sync(0xffffffffu, a[q], o);
    if ((threadIdx.x & 31) == 0) red[q][threadIdx.x >> 5] = a[q];
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double t = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) t += red[threadIdx.x][w];
    partial[threadIdx.x * gridDim.x + blockIdx.x] = t;
  }
}

int blocks_for(long long n, int sms) {
  const long long b = (n + kThreads - 1) / kThreads;
  return (int)std::max<long long>(1, std::min<long long>(b, (long long)sms * 8));
}

// RAII device buffer for the generator's transient workspace
struct DevBuf {
  void* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  cudaError_t alloc(size_t bytes) { return cudaMalloc(&p, bytes); }
};
struct Plan {
  cufftHandle h = 0;
  bool ok = false;
  ~Plan() {
    if (ok) cufftDestroy(h);
  }
};

int cufft_rc(cufftResult r) {
  using host::last_cuda_error;
  if (r == CUFFT_SUCCESS) return PMFMHD_OK;
  last_cuda_error() = "cuFFT error " + std::to_string((int)r);
  return PMFMHD_ECUDA;
}

}  // namespace
}  // namespace pmf

using namespace pmf;
using namespace pmf::host;

extern "C" {

int pmfmhd_pmf_batchelor_field(pmfmhd_ctx* c, const pmfmhd_pmf_params* p, float* const B[3], double stats[6],
                               void* stream) {
  if (c == nullptr || p == nullptr || B == nullptr || !B[0] || !B[1] || !B[2]) return PMFMHD_EINVAL;
  const int nx = p->nx, ny = p->ny, nz = p->nz;
  if (nx < 2 || ny < 1 || nz < 1) return PMFMHD_ESHAPE;
  if (nx % 2 != 0) return PMFMHD_ESHAPE;  // rfft packing needs even nx (pmf.jl:318)
  if (p->realization != PMFMHD_PMF_HASH && p->realization != PMFMHD_PMF_HASH_ZERO_PHASE)
    return PMFMHD_EUNSUPPORTED;
  const int mind = std::min(nx, std::min(ny, nz));
  const double L = p->box;
  if (!(L > 0.0) || !(p->brms > 0.0)) return PMFMHD_EINVAL;
  if (p->invariant_axis < 0 || p->invariant_axis > 3) return PMFMHD_EINVAL;
  const double RL = p->realization_box > 0.0 ? p->realization_box : L;
  if (!(RL + 32 * DBL_EPSILON * std::max(1.0, RL) >= L)) return PMFMHD_EINVAL;
  const double ratio = RL / L;
  const long long qscale = std::llround(ratio);
  if (!(qscale > 0 && std::fabs(ratio - (double)qscale) <= 32 * DBL_EPSILON * std::max(1.0, std::fabs(ratio))))
    return PMFMHD_EINVAL;  // reference_box / box must be a positive integer (pmf.jl:153-157)
  const double kc = p->kcut > 0.0 ? p->kcut : M_PI * mind / L;
  if (!(kc > 0.0) || !(p->kmin >= 0.0)) return PMFMHD_EINVAL;
  const double km = (p->kmax > 0.0) ? p->kmax : INFINITY;
  if (!(p->kmin < km)) return PMFMHD_EINVAL;
  if (p->minimum_cells_per_wavelength > 0.0) {
    if (!std::isfinite(km)) return PMFMHD_EINVAL;
    const double resolved = 2 * M_PI * mind / (L * p->minimum_cells_per_wavelength);
    if (!(km <= resolved * (1 + 16 * DBL_EPSILON))) return PMFMHD_EINVAL;
  }
  const bool preserve_low = p->preserve_low_kmax > 0.0;
  if (preserve_low && !(p->preserve_low_kmax <= km)) return PMFMHD_EINVAL;
  const double low_kc = p->preserve_low_kcut > 0.0 ? p->preserve_low_kcut : kc;
  int norm = p->normalization;  // 0 auto, 1 total band, 2 reference band (pmf.jl:28-39)
  if (norm == 0) norm = preserve_low ? 2 : 1;
  if (norm != 1 && norm != 2) return PMFMHD_EINVAL;
  if (norm == 2 && !preserve_low) return PMFMHD_EINVAL;
  if (p->curl_symbol != 0 && p->curl_symbol != 1) return PMFMHD_EINVAL;
  const int cref = p->curl_reference_n;
  if (cref != 0 && (p->curl_symbol != 0 || cref < 0 || cref > mind)) return PMFMHD_EINVAL;
  // source grids of the high and the preserved low band (mode locking, pmf.jl:368-402)
  const int source_lock = p->high_mode_lock_n != 0 ? p->high_mode_lock_n : (!preserve_low ? p->mode_lock_n : 0);
  int sx_ = nx, sy_ = ny, sz_ = nz;
  if (source_lock != 0 && source_lock != mind) {
    if (source_lock < 0 || source_lock > mind || !(km <= M_PI * source_lock / L)) return PMFMHD_EINVAL;
    sx_ = sy_ = sz_ = source_lock;
  }
  int lx_ = nx, ly_ = ny, lz_ = nz;
  if (preserve_low && p->mode_lock_n != 0 && p->mode_lock_n != mind) {
    const int l = p->mode_lock_n;
    if (l < 0 || l > mind || !(p->preserve_low_kmax <= M_PI * l / L)) return PMFMHD_EINVAL;
    lx_ = ly_ = lz_ = l;
  }
  const double vt = (double)nx * ny * nz;
  const bool hi_same = sx_ == nx && sy_ == ny && sz_ == nz;
  const bool lo_same = lx_ == nx && ly_ == ny && lz_ == nz;
  if ((!hi_same && sx_ % 2 != 0) || (!lo_same && lx_ % 2 != 0)) return PMFMHD_ESHAPE;

  PmfModes P{};
  P.nx = nx; P.ny = ny; P.nz = nz; P.nxh = nx / 2 + 1;
  P.seed = p->seed;
  P.qscale = (int)qscale;
  P.zero_phase = p->realization == PMFMHD_PMF_HASH_ZERO_PHASE;
  P.two_pi_over_L = (2.0 * M_PI) / L;
  P.km2 = km * km;
  P.kmin2 = p->kmin * p->kmin;
  P.kc = kc;
  P.low_kc = low_kc;
  if (preserve_low) {
    const float lk = (float)p->preserve_low_kmax;
    const float thr = (lk * lk) * (1.0f + 8.0f * FLT_EPSILON);
    P.low_thr = (double)thr;
  } else {
    P.low_thr = -1.0;
  }
  P.amp_exp = 0.5 * (p->energy_index - 4.0);
  P.order = p->cutoff_order;
  P.energy_index = p->energy_index;
  P.high_source_scale =
      preserve_low ? (float)std::sqrt(((double)sx_ * sy_ * sz_) / ((double)lx_ * ly_ * lz_)) : 1.0f;
  P.invariant_axis = p->invariant_axis;
  P.fixed_power = p->fixed_mode_power != 0;
  P.project = cref != 0 && cref != mind;
  P.high = Source{sx_, sy_, sz_, hi_same, (float)(vt / ((double)sx_ * sy_ * sz_))};
  P.low = Source{lx_, ly_, lz_, lo_same, (float)(vt / ((double)lx_ * ly_ * lz_))};

  // derivative symbols: Float32 of sin(k dx)/dx (centred) or k (continuum), target and
  // reference grid (pmf.jl:438-449)
  const int nxh = P.nxh;
  std::vector<float> sym(2 * (size_t)(nxh + ny + nz));
  const double dx = L / nx, rdx = cref == 0 ? dx : L / cref;
  auto kof = [&](int idx, int n, bool half) { return (double)(half ? idx : (idx <= n / 2 ? idx : idx - n)) * P.two_pi_over_L; };
  auto symb = [&](double k, double h) { return (float)(p->curl_symbol == 0 ? std::sin(k * h) / h : k); };
  size_t o = 0;
  for (int pass = 0; pass < 2; ++pass) {
    const double h = pass == 0 ? dx : rdx;
    for (int i = 0; i < nxh; ++i) sym[o++] = symb(kof(i, nx, true), h);
    for (int j = 0; j < ny; ++j) sym[o++] = symb(kof(j, ny, false), h);
    for (int k = 0; k < nz; ++k) sym[o++] = symb(kof(k, nz, false), h);
  }

  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const long long n = (long long)nx * ny * nz;
  const long long nck = (long long)nxh * ny * nz;
  DevBuf dsym, dbk, dlk, dtmp, dpart, dres;
  PMF_CK(dsym.alloc(sym.size() * sizeof(float)));
  PMF_CK(cudaMemcpyAsync(dsym.p, sym.data(), sym.size() * sizeof(float), cudaMemcpyHostToDevice, s));
  PMF_CK(dbk.alloc(3 * (size_t)nck * sizeof(float2)));
  if (preserve_low) PMF_CK(dlk.alloc(3 * (size_t)nck * sizeof(float2)));
  // cuFFT writes only to this scratch: its own allocation is aligned for the transform, while
  // the caller's field arrays may sit at any float offset of a packed state
  PMF_CK(dtmp.alloc((size_t)n * sizeof(float)));
  const int nb = blocks_for(n, c->sms);
  PMF_CK(dpart.alloc((size_t)nb * sizeof(double)));
  PMF_CK(dres.alloc(16 * sizeof(double)));
  P.sym = static_cast<const float*>(dsym.p);
  float2* bk = static_cast<float2*>(dbk.p);
  float2* lk = preserve_low ? static_cast<float2*>(dlk.p) : nullptr;
  pmf_modes_kernel<<<blocks_for(nck, c->sms), kThreads, 0, s>>>(P, bk, lk);
  PMF_CK(cudaGetLastError());

  Plan plan;
  int rc = cufft_rc(cufftPlan3d(&plan.h, nz, ny, nx, CUFFT_C2R));
  if (rc) return rc;
  plan.ok = true;
  if ((rc = cufft_rc(cufftSetStream(plan.h, s)))) return rc;
  const float inv_n = (float)(1.0 / vt);  // FFTW's irfft is normalised
  double* res = static_cast<double*>(dres.p);
  double* part = static_cast<double*>(dpart.p);
  float* tmp = static_cast<float*>(dtmp.p);
  for (int d = 0; d < 3; ++d) {
    if ((rc = cufft_rc(cufftExecC2R(plan.h, reinterpret_cast<cufftComplex*>(bk + d * nck), tmp)))) return rc;
    scale_sumsq_kernel<<<nb, kThreads, 0, s>>>(tmp, B[d], n, inv_n, true, part);
    fold_kernel<<<1, 1, 0, s>>>(part, nb, res, d);
    if (preserve_low) {
      if ((rc = cufft_rc(cufftExecC2R(plan.h, reinterpret_cast<cufftComplex*>(lk + d * nck), tmp)))) return rc;
      scale_sumsq_kernel<<<nb, kThreads, 0, s>>>(tmp, tmp, n, inv_n, false, part);
      fold_kernel<<<1, 1, 0, s>>>(part, nb, res, 3 + d);
    }
  }
  PMF_CK(cudaGetLastError());
  double h[6] = {0, 0, 0, 0, 0, 0};
  PMF_CK(cudaMemcpyAsync(h, res, 6 * sizeof(double), cudaMemcpyDeviceToHost, s));
  PMF_CK(cudaStreamSynchronize(s));
  const double rms0 = std::sqrt((h[0] + h[1] + h[2]) / vt);
  if (!(rms0 > 0.0)) return PMFMHD_EINADMISSIBLE;  // zero field: check kcut, kmax and dims
  const double ref_rms0 = preserve_low ? std::sqrt((h[3] + h[4] + h[5]) / vt) : rms0;
  if (!(ref_rms0 > 0.0)) return PMFMHD_EINADMISSIBLE;
  const float scale = (float)(p->brms / (norm == 2 ? ref_rms0 : rms0));
  for (int d = 0; d < 3; ++d) {
    scale_sumsq_kernel<<<nb, kThreads, 0, s>>>(B[d], B[d], n, scale, true, part);
    fold_kernel<<<1, 1, 0, s>>>(part, nb, res, 6 + d);
  }
  PMF_CK(cudaGetLastError());
  double t[3];
  PMF_CK(cudaMemcpyAsync(t, res + 6, 3 * sizeof(double), cudaMemcpyDeviceToHost, s));
  PMF_CK(cudaStreamSynchronize(s));
  if (stats) {
    const double total = std::sqrt((t[0] + t[1] + t[2]) / vt);
    const double refb = (double)scale * ref_rms0;
    stats[0] = total;
    stats[1] = refb;
    stats[2] = norm == 2 ? refb : total;
    stats[3] = kc;
    stats[4] = km;
    stats[5] = (double)P.high_source_scale;
  }
  return PMFMHD_OK;
}

int pmfmhd_periodic_tile(pmfmhd_ctx* c, const float* src, int sx, int sy, int sz, float* dst, int nx, int ny, int nz,
                         void* stream) {
  if (c == nullptr || src == nullptr || dst == nullptr) return PMFMHD_EINVAL;
  if (sx < 1 || sy < 1 || sz < 1 || nx < 1 || ny < 1 || nz < 1) return PMFMHD_ESHAPE;
  if (nx % sx || ny % sy || nz % sz) return PMFMHD_ESHAPE;  // the tile must divide the grid
  const long long n = (long long)nx * ny * nz;
  tile_kernel<<<blocks_for(n, c->sms), kThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(src, sx, sy, sz, dst,
                                                                                              nx, ny, n);
  PMF_CK(cudaGetLastError());
  return PMFMHD_OK;
}

int pmfmhd_pmf_install(pmfmhd_ctx* c, const pmfmhd_grid* g, float* const U[9], float rho0, float p0, void* stream) {
  if (c == nullptr) return PMFMHD_EINVAL;
  int rc = check_grid(g);
  if (rc) return rc;
  if (U == nullptr) return PMFMHD_EINVAL;
  for (int f = 0; f < 9; ++f)
    if (U[f] == nullptr) return PMFMHD_EINVAL;
  if (!std::isfinite(rho0) || !std::isfinite(p0)) return PMFMHD_EINVAL;
  const long long n = ncells(g);
  const float eth = p0 / (g->gamma - 1.0f);
  pmf_install_kernel<<<blocks_for(n, c->sms), kThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      U[0], U[1], U[2], U[3], U[4], U[5], U[6], U[7], U[8], n, rho0, eth);
  PMF_CK(cudaGetLastError());
  return PMFMHD_OK;
}

int pmfmhd_ct_faces_from_cells(pmfmhd_ctx* c, const pmfmhd_grid* g, float* const U[9], float* ct, double stats[3],
                               void* stream) {
  if (c == nullptr || ct == nullptr) return PMFMHD_EINVAL;
  int rc = check_grid(g);
  if (rc) return rc;
  if (!all_periodic(g)) return PMFMHD_EUNSUPPORTED;
  if (U == nullptr) return PMFMHD_EINVAL;
  for (int f = 0; f < 9; ++f)
    if (U[f] == nullptr) return PMFMHD_EINVAL;
  const int nx = g->nx, ny = g->ny, nz = g->nz, nxh = nx / 2 + 1;
  const long long n = ncells(g), nck = (long long)nxh * ny * nz;
  const long long n2 = (n + 1) & ~1LL;  // component stride: every component 16-byte aligned for cuFFT
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  DevBuf dold, dbh, dface, dpart, dres;
  PMF_CK(dold.alloc(3 * (size_t)n2 * sizeof(double)));
  PMF_CK(dbh.alloc(3 * (size_t)nck * sizeof(double2)));
  PMF_CK(dface.alloc((size_t)n * sizeof(double)));
  const int nb = blocks_for(n, c->sms);
  PMF_CK(dpart.alloc(3 * (size_t)nb * sizeof(double)));
  PMF_CK(dres.alloc(4 * sizeof(double)));
  double* old = static_cast<double*>(dold.p);
  double2* bh = static_cast<double2*>(dbh.p);
  for (int d = 0; d < 3; ++d) to_double_kernel<<<nb, kThreads, 0, s>>>(U[5 + d], old + d * n2, n);
  PMF_CK(cudaGetLastError());
  Plan fwd, inv;
  if ((rc = cufft_rc(cufftPlan3d(&fwd.h, nz, ny, nx, CUFFT_D2Z)))) return rc;
  fwd.ok = true;
  if ((rc = cufft_rc(cufftPlan3d(&inv.h, nz, ny, nx, CUFFT_Z2D)))) return rc;
  inv.ok = true;
  if ((rc = cufft_rc(cufftSetStream(fwd.h, s))) || (rc = cufft_rc(cufftSetStream(inv.h, s)))) return rc;
  for (int d = 0; d < 3; ++d)
    if ((rc = cufft_rc(cufftExecD2Z(fwd.h, old + d * n2, reinterpret_cast<cufftDoubleComplex*>(bh + d * nck)))))
      return rc;
  ct_face_modes_kernel<<<blocks_for(nck, c->sms), kThreads, 0, s>>>(bh, nx, ny, nz);
  PMF_CK(cudaGetLastError());
  double* face = static_cast<double*>(dface.p);
  for (int d = 0; d < 3; ++d) {
    if ((rc = cufft_rc(cufftExecZ2D(inv.h, reinterpret_cast<cufftDoubleComplex*>(bh + d * nck), face)))) return rc;
    faces_to_float_kernel<<<nb, kThreads, 0, s>>>(face, ct + (size_t)d * n, n, 1.0 / (double)n);
  }
  PMF_CK(cudaGetLastError());
  if ((rc = pmfmhd_ct_install_faces(c, g, U, ct, stream))) return rc;
  double* part = static_cast<double*>(dpart.p);
  ct_change_kernel<<<nb, kThreads, 0, s>>>(U[5], U[6], U[7], old, old + n2, old + 2 * n2, n, part);
  for (int q = 0; q < 3; ++q) fold_kernel<<<1, 1, 0, s>>>(part + q * nb, nb, static_cast<double*>(dres.p), q);
  PMF_CK(cudaGetLastError());
  double h[3];
  PMF_CK(cudaMemcpyAsync(h, dres.p, 3 * sizeof(double), cudaMemcpyDeviceToHost, s));
  PMF_CK(cudaStreamSynchronize(s));
  if (stats) {
    double divb = 0.0;
    if ((rc = pmfmhd_max_divb_face(c, g, ct, &divb, stream))) return rc;
    const double brms = std::sqrt(h[2] / (double)n);
    stats[0] = h[1] > 0.0 ? std::sqrt(h[0] / h[1]) : 0.0;
    stats[1] = h[1] > 0.0 ? h[2] / h[1] : 1.0;
    stats[2] = brms > 0.0 ? divb * g->dx / brms : 0.0;
  }
  return PMFMHD_OK;
}

}  // extern "C"
