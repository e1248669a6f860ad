// Host-side view of the step-kernel instantiations.
#pragma once
#include <cstddef>

namespace pmf {
struct StepArgs;
struct BoxStep;
using StepKernel = void (*)(const StepArgs);
using BatchKernel = void (*)(const BoxStep*, int, long long);

struct StepKernelInfo {
  StepKernel fn;      // null if the combination is not instantiated
  size_t smem_bytes;  // dynamic shared memory per CTA
  int threads;        // threads per CTA
};

// Rows per CTA that are instantiated (tile candidates for the autotuner).
constexpr int kTileRows[] = {5, 8, 9, 13};
constexpr int kNumTileRows = 4;

// `src`: SRC_NONE, or a source-coupled step (SRC_DRAG, SRC_RAD; `comp` must be false).
StepKernelInfo step_kernel_info(int ty, int recon, int rsol, bool ct, bool comp, int src = 0);
// The many-box form of the same kernel (same shared memory and block size).
BatchKernel batch_kernel(int ty, int recon, int rsol, bool ct, bool comp);
// The HLLD census step (8 owned rows, MC-PLM, GLM, plain update).
StepKernelInfo step_census_kernel_info();
constexpr int kCensusRows = 8;
}  // namespace pmf
