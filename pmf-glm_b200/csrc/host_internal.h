// Host-side internals shared by the C-ABI translation units (not part of the public ABI).
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

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

int check_grid(const pmfmhd_grid* g);
bool all_periodic(const pmfmhd_grid* g);
Phys phys_of(const pmfmhd_grid* g);
long long ncells(const pmfmhd_grid* g);
int occupancy_of(const StepKernelInfo& k);

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
  std::mutex mu;
};

namespace pmf {
namespace host {
Tune tune_for(pmfmhd_ctx* c, const pmfmhd_grid* g, bool ct, bool comp);
int aux_blocks(const pmfmhd_ctx* c, long long nc);
}  // namespace host
}  // namespace pmf
