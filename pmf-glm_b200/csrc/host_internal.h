// Host-side internals shared by the C-ABI translation units (not part of the public ABI).
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include <cuda.h>

#include "../../include/pmfmhd.h"
#include "dispatch.h"
#include "physics.cuh"

namespace pmf {
namespace host {

// Text of the last CUDA error on this thread (pmfmhd_last_cuda_error).
std::string& last_cuda_error();

#define PMF_CK(call)                                                              \
  do {                                                                            \
    cudaError_t e_ = (call);                                                      \
    if (e_ != cudaSuccess) {                                                      \
      ::pmf::host::last_cuda_error() = std::string(#call) + ": " + cudaGetErrorString(e_); \
      return PMFMHD_ECUDA;                                                        \
    }                                                                             \
  } while (0)

struct TuneKey {
  int nx, ny, nz, ct, comp, recon, rsol;
  bool operator<(const TuneKey& o) const {
    return std::tie(nx, ny, nz, ct, comp, recon, rsol) < std::tie(o.nx, o.ny, o.nz, o.ct, o.comp, o.recon, o.rsol);
  }
};
// Tile height and the minimum number of planes per CTA.
struct Tune {
  int ty, tz;
};
struct GraphEntry {
  std::vector<unsigned char> key;
  cudaGraphExec_t exec;
};

struct MapKey {
  const void* ptr;
  int nx, ny, nz, ty;
  bool operator<(const MapKey& o) const {
    return std::tie(ptr, nx, ny, nz, ty) < std::tie(o.ptr, o.nx, o.ny, o.nz, o.ty);
  }
};

int check_grid(const pmfmhd_grid* g);
bool all_periodic(const pmfmhd_grid* g);
Phys phys_of(const pmfmhd_grid* g);
long long ncells(const pmfmhd_grid* g);
int occupancy_of(const StepKernelInfo& k);

}  // namespace host
}  // namespace pmf

namespace pmf {
namespace host {
// Workspace of the host-buffer step (pmfmhd_step_glm_host): device copies of the state in and
// out, three streams (copy in, compute, copy out) and per-chunk events, created on first use.
struct HostPath {
  float* dev = nullptr;     // 18 * cells floats: U then Unew
  size_t floats = 0;
  cudaStream_t s[3] = {nullptr, nullptr, nullptr};
  std::vector<cudaEvent_t> ev;  // 3 per chunk: arrived, computed, copied out
  cudaEvent_t start = nullptr;
};
}  // namespace host
}  // namespace pmf

struct pmfmhd_ctx {
  int device = 0;
  int sms = 148;
  unsigned int* d_smax = nullptr;           // bits of the last step's max signal speed
  unsigned long long* d_u64 = nullptr;      // bits of an FP64 max
  double* d_partial = nullptr;              // totals partials
  double* d_tot = nullptr;                  // totals
  unsigned char* h_pin = nullptr;           // pinned host landing area
  cudaStream_t cap = nullptr;               // stream used to record graphs
  std::map<pmf::host::TuneKey, pmf::host::Tune> tune;
  std::vector<pmf::host::GraphEntry> graphs;
  std::map<pmf::host::MapKey, CUtensorMap> maps;  // TMA descriptors of field arrays
  unsigned int* d_status = nullptr;                // device status bits of the step kernels
  pmf::host::HostPath hp;                          // host-buffer step workspace
  int tma_stall_polls = 0;                         // pmfmhd_set_tma_stall test hook
  float* d_mask = nullptr;                         // copy of a radiation fallback mask (masked step
  long long mask_cells = 0;                        // with density tracking), allocated on first use
  std::mutex mu;
};

namespace pmf {
namespace host {
Tune tune_for(pmfmhd_ctx* c, const pmfmhd_grid* g, bool ct, bool comp);
// Tensor maps for the nine fields U (box PLANE_W x (ty+4) x 1); false if TMA cannot be used
// for this grid (x extent not a multiple of 4, unaligned pointers, box larger than the grid).
bool field_maps(pmfmhd_ctx* c, const pmfmhd_grid* g, const float* const U[9], int ty, CUtensorMap out[9]);
int aux_blocks(const pmfmhd_ctx* c, long long nc);
// Drag coefficients of one step with impulse q toward `v0` (null: at rest), FP32.
DragCoef drag_coefficients(float q, const float* v0);
}  // namespace host
}  // namespace pmf
