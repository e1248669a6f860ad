// Allocation-free FP64 conserved totals: pmfmhd_conserved_totals_noalloc.
//
// Some callers cannot call cudaMalloc at all: code running inside a host that owns the
// device memory pool (a Julia/CUDA.jl session whose allocator must see every allocation,
// a plugin loaded into another application, a process that has reserved all free memory
// for its state), or code that must not allocate between steps. For them this entry point
// needs no context and allocates nothing: its scratch (one FP64 partial sum per field per
// 256-cell block, plus the 8 results) is a file-scope __device__ array in this library,
// 4 MiB, that every GPU which loads the library holds until the process exits.
//
// Limits and behaviour:
//   * at most kMaxCells = 2^24 cells (256^3); larger grids are rejected with
//     PMFMHD_ESHAPE before any device work;
//   * one partial per block of 256 consecutive cells, summed in a fixed order, so the bits
//     of the result do not depend on the GPU's SM count;
//   * every call shares the one array and leaves its contents behind; each call overwrites
//     every partial it reads, so nothing needs clearing first, but calls that overlap on
//     the GPU (two streams, two host threads) race on it and must be serialised;
//   * the first call in a CUDA context looks up the array's device address with that
//     context current (cudaGetSymbolAddress) and caches it with the context's unique id. The
//     array lives in the library's module, which is loaded again whenever a context is
//     re-created (after cudaDeviceReset, or when the host application rebuilds the primary
//     context), possibly at another address; a call that finds another context current than
//     the cached one looks the address up again. Make the first call of each context before
//     any stream capture is active.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <mutex>

#include "../../include/pmfmhd.h"

namespace {

constexpr int kBlock = 256;
constexpr long long kMaxCells = 1LL << 24;
constexpr int kMaxPartials = (int)(kMaxCells / kBlock);  // 65536
constexpr int kMaxDevices = 64;

struct FieldPtrs {
  const float* p[9];
};

// [kMaxPartials][8] partial sums followed by the 8 results
static __device__ __align__(256) double g_totals_scratch[kMaxPartials * 8 + 8];

// Device address of g_totals_scratch per device, valid in the context with id ctx_id.
struct ScratchAddr {
  unsigned long long ctx_id;
  double* ptr;
};
std::mutex g_mu;
ScratchAddr g_scratch_addr[kMaxDevices] = {};

// Unique id of the calling thread's current context (cuCtxGetId: unique for the life of the
// process, so a re-created context never repeats an old id), or 0 if there is no current
// context or the driver entry points are unavailable. Reached through the runtime's driver
// entry points (no link to libcuda).
unsigned long long current_context_id() {
  static PFN_cuCtxGetCurrent_v4000 get_current = nullptr;
  static PFN_cuCtxGetId_v12000 get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(p);
    p = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<PFN_cuCtxGetId_v12000>(p);
  });
  if (get_current == nullptr || get_id == nullptr) return 0;
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr) return 0;
  unsigned long long id = 0;
  if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

__global__ void __launch_bounds__(kBlock) totals_block_kernel(const FieldPtrs U, int nc, double* part) {
  __shared__ double red[8][kBlock / 32];
  const int c = blockIdx.x * kBlock + threadIdx.x;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    double v = c < nc ? (double)__ldg(U.p[q] + c) : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) red[q][w] = v;
  }
  __syncthreads();
  if (threadIdx.x < 8) {
    double t = 0.0;
    for (int i = 0; i < kBlock / 32; ++i) t += red[threadIdx.x][i];
    part[(size_t)blockIdx.x * 8 + threadIdx.x] = t;
  }
}

__global__ void __launch_bounds__(kBlock) totals_fold_kernel(const double* part, int nparts, double scale,
                                                             double* out) {
  __shared__ double red[8][kBlock];
  const int t = threadIdx.x;
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    double s = 0.0;
    for (int i = t; i < nparts; i += kBlock) s += part[(size_t)i * 8 + q];
    red[q][t] = s;
  }
  __syncthreads();
  for (int h = kBlock / 2; h > 0; h >>= 1) {
    if (t < h) {
#pragma unroll
      for (int q = 0; q < 8; ++q) red[q][t] += red[q][t + h];
    }
    __syncthreads();
  }
  if (t < 8) out[t] = red[t][0] * scale;
}

}  // namespace

extern "C" int pmfmhd_conserved_totals_noalloc(const pmfmhd_grid* g, const float* const U[9], double out[8],
                                               void* stream) {
  if (g == nullptr || U == nullptr || out == nullptr) return PMFMHD_EINVAL;
  for (int f = 0; f < 8; ++f)
    if (U[f] == nullptr) return PMFMHD_EINVAL;
  if (g->nx < 1 || g->ny < 1 || g->nz < 1) return PMFMHD_ESHAPE;
  if (!(g->dx > 0.0f) || !std::isfinite(g->dx)) return PMFMHD_EINVAL;
  const long long nc = (long long)g->nx * g->ny * g->nz;
  if (nc > kMaxCells) return PMFMHD_ESHAPE;  // beyond the static scratch: rejected, no work done
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return PMFMHD_ECUDA;
  double* scratch;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    ScratchAddr& slot = g_scratch_addr[dev];
    const unsigned long long id = current_context_id();
    if (slot.ptr == nullptr || id == 0 || id != slot.ctx_id) {
      // set-up in this context: look the array's address up with the device current (this
      // also creates the primary context if none is current yet), then record whose it is
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_totals_scratch) != cudaSuccess || p == nullptr) return PMFMHD_ECUDA;
      slot.ptr = static_cast<double*>(p);
      slot.ctx_id = current_context_id();  // 0 if unknown: the next call looks it up again
    }
    scratch = slot.ptr;
  }
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  FieldPtrs u;
  for (int f = 0; f < 9; ++f) u.p[f] = U[f];
  const int nparts = (int)((nc + kBlock - 1) / kBlock);
  totals_block_kernel<<<nparts, kBlock, 0, s>>>(u, (int)nc, scratch);
  const float dV = g->dx * g->dx * g->dx;  // dx^3 in FP32, as the reference (diagnostics.jl:45)
  double* res = scratch + (size_t)kMaxPartials * 8;
  totals_fold_kernel<<<1, kBlock, 0, s>>>(scratch, nparts, (double)dV, res);
  if (cudaGetLastError() != cudaSuccess) return PMFMHD_ECUDA;
  if (cudaMemcpyAsync(out, res, 8 * sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess) return PMFMHD_ECUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return PMFMHD_ECUDA;
  return PMFMHD_OK;
}
