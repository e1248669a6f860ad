// C ABI of libpmfmhd.so: argument checks, tile selection, launches, CUDA-graph replay of
// fixed-dt step sequences, and the FP64 diagnostics. See include/pmfmhd.h.
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/pmfmhd.h"
#include "aux_kernels.cuh"
#include "dispatch.h"
#include "host_internal.h"
#include "step_kernel.cuh"

using namespace pmf;
using namespace pmf::host;

namespace {
constexpr int kTotBlocksMax = 1024;
}  // namespace

namespace pmf {
namespace host {
std::string& last_cuda_error() {
  thread_local std::string e;
  return e;
}
}  // namespace host
}  // namespace pmf

namespace pmf {
namespace host {

cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

int check_grid(const pmfmhd_grid* g) {
  if (g == nullptr) return PMFMHD_EINVAL;
  if (g->nx < 1 || g->ny < 1 || g->nz < 1) return PMFMHD_ESHAPE;
  const long long nc = (long long)g->nx * g->ny * g->nz;
  if (nc >= (1LL << 31)) return PMFMHD_ESHAPE;
  for (int d = 0; d < 3; ++d)
    if (g->bc[d] < 0 || g->bc[d] > 2) return PMFMHD_EINVAL;
  if (g->recon < 0 || g->recon > 2 || g->riemann < 0 || g->riemann > 2) return PMFMHD_EINVAL;
  if (!(g->dx > 0.0f) || !std::isfinite(g->dx) || !(g->gamma > 1.0f) || !std::isfinite(g->gamma))
    return PMFMHD_EINVAL;
  if (!std::isfinite(g->smallr) || !std::isfinite(g->pfl) || !std::isfinite(g->llf_dmin) ||
      !std::isfinite(g->llf_pmin))
    return PMFMHD_EINVAL;
  if (!std::isfinite(g->hlld_dtol_rel) || !(g->hlld_dtol_rel >= 0.0f)) return PMFMHD_EINVAL;
  return PMFMHD_OK;
}
bool all_periodic(const pmfmhd_grid* g) {
  return g->bc[0] == BC_PERIODIC && g->bc[1] == BC_PERIODIC && g->bc[2] == BC_PERIODIC;
}
template <class P> bool nonnull(P* const* v, int n) {
  if (v == nullptr) return false;
  for (int i = 0; i < n; ++i)
    if (v[i] == nullptr) return false;
  return true;
}
// resid is either NULL / all-NULL (plain update) or 7 non-null pointers
int resid_mode(float* const* r, bool* comp) {
  *comp = false;
  if (r == nullptr) return PMFMHD_OK;
  int n = 0;
  for (int i = 0; i < 7; ++i) n += r[i] != nullptr;
  if (n == 0) return PMFMHD_OK;
  if (n != 7) return PMFMHD_EINVAL;
  *comp = true;
  return PMFMHD_OK;
}
Phys phys_of(const pmfmhd_grid* g) {
  return Phys{g->gamma, g->smallr, g->pfl, g->llf_dmin, g->llf_pmin, g->hlld_dtol_rel};
}
long long ncells(const pmfmhd_grid* g) { return (long long)g->nx * g->ny * g->nz; }
int aux_blocks(const pmfmhd_ctx* c, long long nc) {
  long long b = (nc + AUX_THREADS - 1) / AUX_THREADS;
  long long cap = (long long)c->sms * 8;
  return (int)(b < cap ? (b < 1 ? 1 : b) : cap);
}

// Tile height and the minimum number of planes per CTA (the launch gives every CTA an
// equal share of the (column, plane) space, but never less than `tz` planes).
Tune default_tune(const pmfmhd_ctx*, const pmfmhd_grid* g) {
  Tune t;
  t.ty = g->ny >= 8 ? 8 : 5;
  t.tz = 16;
  return t;
}

Tune tune_for(pmfmhd_ctx* c, const pmfmhd_grid* g, bool ct, bool comp) {
  std::lock_guard<std::mutex> lk(c->mu);
  auto it = c->tune.find(TuneKey{g->nx, g->ny, g->nz, ct, comp, g->recon, g->riemann});
  if (it != c->tune.end()) return it->second;
  return default_tune(c, g);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link to libcuda).
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

bool field_maps(pmfmhd_ctx* c, const pmfmhd_grid* g, const float* const U[9], int ty, CUtensorMap out[9]) {
  auto enc = encode_fn();
  if (enc == nullptr || g->nx % 4 != 0 || g->nx < PLANE_W || g->ny < ty + 4) return false;
  for (int f = 0; f < 9; ++f)
    if (reinterpret_cast<uintptr_t>(U[f]) % 16 != 0) return false;
  std::lock_guard<std::mutex> lk(c->mu);
  for (int f = 0; f < 9; ++f) {
    const MapKey key{U[f], g->nx, g->ny, g->nz, ty};
    auto it = c->maps.find(key);
    if (it != c->maps.end()) {
      out[f] = it->second;
      continue;
    }
    const cuuint64_t dims[3] = {(cuuint64_t)g->nx, (cuuint64_t)g->ny, (cuuint64_t)g->nz};
    const cuuint64_t strides[2] = {(cuuint64_t)g->nx * 4, (cuuint64_t)g->nx * g->ny * 4};
    const cuuint32_t box[3] = {(cuuint32_t)PLANE_W, (cuuint32_t)(ty + 4), 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUtensorMap m;
    if (enc(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(U[f]), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return false;
    if (c->maps.size() > 4096) c->maps.clear();
    c->maps[key] = m;
    out[f] = m;
  }
  return true;
}

// Resident CTAs per SM of a step kernel (cached per kernel).
int occupancy_of(const StepKernelInfo& k) {
  static std::mutex mu;
  static std::map<const void*, int> cache;
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find((const void*)k.fn);
  if (it != cache.end()) return it->second;
  int occ = 1;
  if (cudaFuncSetAttribute((const void*)k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.smem_bytes) !=
          cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, (const void*)k.fn, k.threads, k.smem_bytes) != cudaSuccess ||
      occ < 1)
    occ = 1;
  cache[(const void*)k.fn] = occ;
  return occ;
}

// `force`: launch this instantiation (its tile height in t.ty) instead of the dispatched one.
int launch_step(pmfmhd_ctx* c, const pmfmhd_grid* g, StepArgs& a, Tune t, bool ct, bool comp,
                cudaStream_t s, int src = SRC_NONE, const StepKernelInfo* force = nullptr) {
  StepKernelInfo k = force ? *force : step_kernel_info(t.ty, g->recon, g->riemann, ct, comp, src);
  if (k.fn == nullptr) return PMFMHD_EUNSUPPORTED;
  const int occ = occupancy_of(k);
  a.nx = g->nx; a.ny = g->ny; a.nz = g->nz;
  for (int d = 0; d < 3; ++d) a.bc[d] = g->bc[d];
  a.ntx = (g->nx + TILE_X - 1) / TILE_X;
  a.nty = (g->ny + t.ty - 1) / t.ty;
  a.P = phys_of(g);
  a.status = c->d_status;
  a.tma_stall_polls = c->tma_stall_polls;
  // Interior planes come in by TMA for the plain and compensated GLM step; the CT and
  // source-coupled instantiations are compiled without the TMA path and stage every plane by
  // per-element cp.async.
  a.use_tma = (!ct && src == SRC_NONE && field_maps(c, g, a.U, t.ty, a.tmap)) ? 1 : 0;
  if (a.zhi <= a.zlo) {  // the whole box unless the caller set a plane range
    a.zlo = 0;
    a.zhi = g->nz;
  }
  const long long Q = (long long)a.ntx * a.nty * (a.zhi - a.zlo);
  const long long slots = (long long)c->sms * occ;
  const long long by_work = std::max<long long>(1, (Q + t.tz - 1) / std::max(1, t.tz));
  const long long blocks = std::min(slots, by_work);
  void* args[] = {(void*)&a};
  PMF_CK(cudaLaunchKernel((const void*)k.fn, dim3((unsigned)blocks), dim3(k.threads), args, k.smem_bytes, s));
  return PMFMHD_OK;
}

void fill_glm_args(StepArgs& a, const float* const U[9], float* const Un[9], float* const resid[7], bool comp,
                   float dtdx, float ch, float decay, unsigned int* smax_bits) {
  std::memset(&a, 0, sizeof(a));
  for (int f = 0; f < 9; ++f) { a.U[f] = U[f]; a.Un[f] = Un[f]; }
  if (comp)
    for (int i = 0; i < 7; ++i) a.resid[i] = resid[i];
  a.dtdx = dtdx; a.ch = ch; a.decay = decay;
  a.smax_bits = smax_bits;
  a.dscal = nullptr;
}

// Drag coefficients of one step with impulse q, in FP32 with the reference's formulas
// (glm_physics.jl:63-66 _drag_phi1, :89-104 _drag_work_coefficients, :115-119 _drag_coefficients).
float drag_phi1(float q) { return std::fabs(q) < 1e-4f ? 1.0f - q / 2.0f + q * q / 6.0f : -std::expm1(-q) / q; }

DragCoef drag_coefficients(float q, const float* v0) {
  DragCoef k;
  for (int c = 0; c < 3; ++c) k.v0[c] = v0 ? v0[c] : 0.0f;
  const float qh = 0.5f * q;
  k.fdecay = std::exp(-qh);
  k.fphi1 = drag_phi1(qh);
  k.decay = std::exp(-q);
  k.phi1 = drag_phi1(q);
  if (q < 0.05f) {
    const float q2 = q * q, q3 = q2 * q, q4 = q3 * q;
    k.A = q * (1.0f - q + (2.0f / 3.0f) * q2 - (1.0f / 3.0f) * q3 + (2.0f / 15.0f) * q4);
    k.C = q * (1.0f - q + (7.0f / 12.0f) * q2 - (1.0f / 4.0f) * q3 + (31.0f / 360.0f) * q4);
    k.D = q * (1.0f / 3.0f - q / 4.0f + (7.0f / 60.0f) * q2 - q3 / 24.0f + (31.0f / 2520.0f) * q4);
  } else {
    const float em1 = -std::expm1(-q), em2 = -std::expm1(-2.0f * q);
    k.A = 0.5f * em2;
    k.C = em1 * em1 / q;
    k.D = (q - 2.0f * em1 + 0.5f * em2) / (q * q);
  }
  return k;
}

// Source terms of a source-coupled step: drag, or radiation coupling (drag + corrections).
struct SourceTerms {
  int src = SRC_NONE;
  DragCoef drag{};
  float* corr = nullptr;
  int rad_flags = 0;
  const float* mask = nullptr;  // masked fallback: the per-cell mask the kernel reads
};

void apply_sources(StepArgs& a, const SourceTerms* st) {
  if (st == nullptr) return;
  a.drag = st->drag;
  a.corr = st->corr;
  a.rad_flags = st->rad_flags;
  a.mask = st->mask;
}

int enqueue_glm(pmfmhd_ctx* c, const pmfmhd_grid* g, const float* const U[9], float* const Un[9], float dt,
                float ch, float decay, float* const resid[7], bool comp, cudaStream_t s, const SourceTerms* st) {
  StepArgs a;
  const float dtdx = dt / g->dx;  // T(dt)/s.dx (integrator_ref.jl:211)
  fill_glm_args(a, U, Un, resid, comp, dtdx, ch, decay, c->d_smax);
  apply_sources(a, st);
  PMF_CK(cudaMemsetAsync(c->d_smax, 0, sizeof(unsigned int), s));
  return launch_step(c, g, a, tune_for(c, g, false, comp), false, comp, s, st ? st->src : SRC_NONE);
}

int enqueue_ct(pmfmhd_ctx* c, const pmfmhd_grid* g, const float* const U[9], float* const Un[9], float* ct, float dt,
               float* const resid[7], bool comp, bool comp_faces, cudaStream_t s, const SourceTerms* st) {
  const long long nc = ncells(g);
  const float dtdx = dt / g->dx;
  StepArgs a;
  fill_glm_args(a, U, Un, resid, comp, dtdx, 0.0f, 1.0f, nullptr);
  apply_sources(a, st);
  for (int d = 0; d < 3; ++d) a.face[d] = ct + (size_t)(CT_BXF + d) * nc;
  for (int k = 0; k < CT_NWORK; ++k) a.work[k] = ct + (size_t)(CT_MFX + k) * nc;
  int rc = launch_step(c, g, a, tune_for(c, g, true, comp), true, comp, s, st ? st->src : SRC_NONE);
  if (rc != PMFMHD_OK) return rc;
  auto sl = [&](int k) { return ct + (size_t)k * nc; };
  const dim3 cg = ctc_grid(g->nx, g->ny, g->nz);
  ct_emf_col_kernel<<<cg, AUX_THREADS, 0, s>>>(sl(CT_MFX), sl(CT_MFY), sl(CT_MFZ), sl(CT_FXBY), sl(CT_FXBZ),
                                               sl(CT_FYBX), sl(CT_FYBZ), sl(CT_FZBX), sl(CT_FZBY), sl(CT_ECX),
                                               sl(CT_ECY), sl(CT_ECZ), sl(CT_EX), sl(CT_EY), sl(CT_EZ), g->nx,
                                               g->ny, g->nz);
  if (comp_faces)
    ct_face_col_kernel<true><<<cg, AUX_THREADS, 0, s>>>(sl(CT_EX), sl(CT_EY), sl(CT_EZ), sl(CT_BXF), sl(CT_BYF),
                                                        sl(CT_BZF), sl(CT_RBX), sl(CT_RBY), sl(CT_RBZ), g->nx,
                                                        g->ny, g->nz, dtdx);
  else
    ct_face_col_kernel<false><<<cg, AUX_THREADS, 0, s>>>(sl(CT_EX), sl(CT_EY), sl(CT_EZ), sl(CT_BXF), sl(CT_BYF),
                                                         sl(CT_BZF), sl(CT_RBX), sl(CT_RBY), sl(CT_RBZ), g->nx,
                                                         g->ny, g->nz, dtdx);
  PMF_CK(cudaMemsetAsync(c->d_smax, 0, sizeof(unsigned int), s));
  MPtr9 un;
  for (int f = 0; f < 9; ++f) un.p[f] = Un[f];
  ct_bcc_col_kernel<<<cg, AUX_THREADS, 0, s>>>(sl(CT_BXF), sl(CT_BYF), sl(CT_BZF), un, g->nx, g->ny, g->nz,
                                               phys_of(g), c->d_smax);
  PMF_CK(cudaGetLastError());
  return PMFMHD_OK;
}

int read_smax(pmfmhd_ctx* c, float* out, cudaStream_t s) {
  PMF_CK(cudaMemcpyAsync(c->h_pin, c->d_smax, sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
  PMF_CK(cudaStreamSynchronize(s));
  unsigned int bits;
  std::memcpy(&bits, c->h_pin, sizeof(bits));
  float v;
  std::memcpy(&v, &bits, sizeof(v));
  *out = v;
  return PMFMHD_OK;
}

}  // namespace host
}  // namespace pmf

extern "C" {

int pmfmhd_version(void) { return 100; }

const char* pmfmhd_strerror(int code) {
  switch (code) {
    case PMFMHD_OK: return "ok";
    case PMFMHD_EINVAL: return "invalid argument";
    case PMFMHD_ESHAPE: return "invalid grid shape";
    case PMFMHD_ECUDA: return "CUDA error";
    case PMFMHD_ETIMEOUT: return "device wait timed out";
    case PMFMHD_EINADMISSIBLE: return "inadmissible state";
    case PMFMHD_ENOMEM: return "out of memory";
    case PMFMHD_EUNSUPPORTED: return "unsupported combination";
  }
  return "unknown error";
}

const char* pmfmhd_last_cuda_error(void) { return last_cuda_error().c_str(); }

int pmfmhd_create(int device, pmfmhd_ctx** out) {
  if (out == nullptr) return PMFMHD_EINVAL;
  *out = nullptr;
  PMF_CK(cudaSetDevice(device));
  pmfmhd_ctx* c = new pmfmhd_ctx();
  c->device = device;
  if (cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) c->sms = 148;
  if (cudaMalloc(&c->d_smax, 256) != cudaSuccess || cudaMalloc(&c->d_u64, 256) != cudaSuccess ||
      cudaMalloc(&c->d_partial, sizeof(double) * 8 * kTotBlocksMax) != cudaSuccess ||
      cudaMalloc(&c->d_tot, sizeof(double) * 8) != cudaSuccess || cudaMallocHost(&c->h_pin, 256) != cudaSuccess ||
      cudaMalloc(&c->d_status, sizeof(unsigned int)) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->cap, cudaStreamNonBlocking) != cudaSuccess) {
    last_cuda_error() = cudaGetErrorString(cudaGetLastError());
    pmfmhd_destroy(c);
    return PMFMHD_ENOMEM;
  }
  PMF_CK(cudaMemset(c->d_smax, 0, 256));
  PMF_CK(cudaMemset(c->d_status, 0, sizeof(unsigned int)));
  *out = c;
  return PMFMHD_OK;
}

int pmfmhd_destroy(pmfmhd_ctx* c) {
  if (c == nullptr) return PMFMHD_OK;
  cudaSetDevice(c->device);
  for (auto& e : c->graphs) cudaGraphExecDestroy(e.exec);
  if (c->cap) cudaStreamDestroy(c->cap);
  cudaFree(c->d_smax);
  cudaFree(c->d_u64);
  cudaFree(c->d_partial);
  cudaFree(c->d_tot);
  cudaFree(c->d_status);
  cudaFreeHost(c->h_pin);
  cudaFree(c->hp.dev);
  cudaFree(c->d_mask);
  for (auto& e : c->hp.ev) cudaEventDestroy(e);
  if (c->hp.start) cudaEventDestroy(c->hp.start);
  for (auto& st : c->hp.s)
    if (st) cudaStreamDestroy(st);
  delete c;
  return PMFMHD_OK;
}

int pmfmhd_step_glm(pmfmhd_ctx* c, const pmfmhd_grid* g, const float* const U[9], float* const Unew[9], float dt,
                    float ch, float decay, float* const resid[7], void* stream) {
  if (c == nullptr) return PMFMHD_EINVAL;
  int rc = check_grid(g);
  if (rc) return rc;
  if (!nonnull(U, 9) || !nonnull(Unew, 9)) return PMFMHD_EINVAL;
  if (!std::isfinite(dt) || !std::isfinite(ch) || !std::isfinite(decay) || !(ch > 0.0f)) return PMFMHD_EINVAL;
  bool comp;
  if ((rc = resid_mode(resid, &comp))) return rc;
  return enqueue_glm(c, g, U, Unew, dt, ch, decay, resid, comp, as_stream(stream), nullptr);
}

int pmfmhd_step_ct(pmfmhd_ctx* c, const pmfmhd_grid* g, const float* const U[9], float* const Unew[9],
                   float* ct_packed, float dt, float* const resid[7], int compensate_faces, void* stream) {
  if (c == nullptr || ct_packed == nullptr) return PMFMHD_EINVAL;
  int rc = check_grid(g);
  if (rc) return rc;
  if (!all_periodic(g)) return PMFMHD_EUNSUPPORTED;
  if (!nonnull(U, 9) || !nonnull(Unew, 9)) return PMFMHD_EINVAL;
  if (!std::isfinite(dt)) return PMFMHD_EINVAL;
  bool comp;
  if ((rc = resid_mode(resid, &comp))) return rc;
  return enqueue_ct(c, g, U, Unew, ct_packed, dt, resid, comp, compensate_faces != 0, as_stream(stream), nullptr);
}

int pmfmhd_step_glm_host(pmfmhd_ctx* c, const pmfmhd_grid* g, const float* const Uh[9], float* const Unh[9],
                         float dt, float ch, float decay, int nchunks, void* stream) {
  if (c == nullptr) return PMFMHD_EINVAL;
  int rc = check_grid(g);
  if (rc) return rc;
  if (!nonnull(Uh, 9) || !nonnull(Unh, 9)) return PMFMHD_EINVAL;
  if (!std::isfinite(dt) || !std::isfinite(ch) || !std::isfinite(decay) || !(ch > 0.0f)) return PMFMHD_EINVAL;
  const int nz = g->nz;
  int C = nchunks > 0 ? nchunks : 16;
  C = std::max(1, std::min(C, nz / 2));  // every chunk at least 2 planes: halos reach chunks c +- 1
  const long long nc = ncells(g), nxy = (long long)g->nx * g->ny;
  HostPath& hp = c->hp;
  const size_t need = 18 * (size_t)nc;
  if (hp.floats < need) {
    cudaFree(hp.dev);
    hp.dev = nullptr;
    hp.floats = 0;
    PMF_CK(cudaMalloc(&hp.dev, need * sizeof(float)));
    hp.floats = need;
  }
  for (auto& st : hp.s)
    if (!st) PMF_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  if (!hp.start) PMF_CK(cudaEventCreateWithFlags(&hp.start, cudaEventDisableTiming));
  while (hp.ev.size() < 3 * (size_t)C) {
    cudaEvent_t e;
    PMF_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    hp.ev.push_back(e);
  }
  cudaStream_t caller = as_stream(stream), sin = hp.s[0], scomp = hp.s[1], sout = hp.s[2];
  const float* Ud[9];
  float* Und[9];
  for (int f = 0; f < 9; ++f) {
    Ud[f] = hp.dev + (size_t)f * nc;
    Und[f] = hp.dev + (size_t)(9 + f) * nc;
  }
  auto zb = [&](int k) { return (int)((long long)nz * k / C); };  // chunk k = planes [zb(k), zb(k+1))
  // host arrays laid out as one (9, cells) block move as one pitched copy per slab
  auto uniform = [&](const float* const* p) {
    for (int f = 1; f < 9; ++f)
      if (p[f] != p[0] + (size_t)f * nc) return false;
    return true;
  };
  const bool in2d = uniform(Uh), out2d = uniform(const_cast<const float* const*>(Unh));
  const size_t pitch = (size_t)nc * sizeof(float);
  auto arrived = [&](int k) { return hp.ev[3 * k]; };
  auto computed = [&](int k) { return hp.ev[3 * k + 1]; };
  // ordered after the caller's prior work
  PMF_CK(cudaEventRecord(hp.start, caller));
  PMF_CK(cudaStreamWaitEvent(sin, hp.start, 0));
  PMF_CK(cudaStreamWaitEvent(scomp, hp.start, 0));
  PMF_CK(cudaStreamWaitEvent(sout, hp.start, 0));
  // copy in: the last chunk first (the periodic lower halo of chunk 0), then 0, 1, ...
  for (int i = 0; i < C; ++i) {
    const int k = (i == 0) ? C - 1 : i - 1;
    const size_t off = (size_t)zb(k) * nxy, len = (size_t)(zb(k + 1) - zb(k)) * nxy;
    if (in2d)
      PMF_CK(cudaMemcpy2DAsync(const_cast<float*>(Ud[0]) + off, pitch, Uh[0] + off, pitch, len * sizeof(float), 9,
                               cudaMemcpyHostToDevice, sin));
    else
      for (int f = 0; f < 9; ++f)
        PMF_CK(cudaMemcpyAsync(const_cast<float*>(Ud[f]) + off, Uh[f] + off, len * sizeof(float),
                               cudaMemcpyHostToDevice, sin));
    PMF_CK(cudaEventRecord(arrived(k), sin));
  }
  // compute chunk k once chunks k-1, k, k+1 (periodic) are resident; copy it out as soon as done
  const float dtdx = dt / g->dx;
  const Tune t = tune_for(c, g, false, false);
  PMF_CK(cudaMemsetAsync(c->d_smax, 0, sizeof(unsigned int), scomp));
  for (int k = 0; k < C; ++k) {
    for (int d = -1; d <= 1; ++d) PMF_CK(cudaStreamWaitEvent(scomp, arrived(((k + d) % C + C) % C), 0));
    StepArgs a;
    fill_glm_args(a, Ud, Und, nullptr, false, dtdx, ch, decay, c->d_smax);
    a.zlo = zb(k);
    a.zhi = zb(k + 1);
    if ((rc = launch_step(c, g, a, t, false, false, scomp))) return rc;
    PMF_CK(cudaEventRecord(computed(k), scomp));
    PMF_CK(cudaStreamWaitEvent(sout, computed(k), 0));
    const size_t off = (size_t)zb(k) * nxy, len = (size_t)(zb(k + 1) - zb(k)) * nxy;
    if (out2d)
      PMF_CK(cudaMemcpy2DAsync(Unh[0] + off, pitch, Und[0] + off, pitch, len * sizeof(float), 9,
                               cudaMemcpyDeviceToHost, sout));
    else
      for (int f = 0; f < 9; ++f)
        PMF_CK(cudaMemcpyAsync(Unh[f] + off, Und[f] + off, len * sizeof(float), cudaMemcpyDeviceToHost, sout));
  }
  PMF_CK(cudaEventRecord(hp.ev[3 * (C - 1) + 2], sout));
  PMF_CK(cudaStreamWaitEvent(caller, hp.ev[3 * (C - 1) + 2], 0));
  PMF_CK(cudaStreamSynchronize(sout));  // the host buffers are complete on return
  return PMFMHD_OK;
}

int pmfmhd_step_glm_drag(pmfmhd_ctx* c, const pmfmhd_grid* g, const float* const U[9], float* const Unew[9],
                         float dt, float ch, float decay, float drag_impulse, const float target_velocity[3],
                         void* stream) {
  if (c == nullptr) return PMFMHD_EINVAL;
  int rc = check_grid(g);
  if (rc) return rc;
  if (!nonnull(U, 9) || !nonnull(Unew, 9)) return PMFMHD_EINVAL;
  if (!std::isfinite(dt) || !std::isfinite(ch) || !std::isfinite(decay) || !(ch > 0.0f)) return PMFMHD_EINVAL;
  if (!std::isfinite(drag_impulse) || !(drag_impulse >= 0.0f)) return PMFMHD_EINVAL;
  SourceTerms st;
  st.src = SRC_DRAG;
  st.drag = drag_coefficients(drag_impulse, target_velocity);
  return enqueue_glm(c, g, U, Unew, dt, ch, decay, nullptr, false, as_stream(stream), &st);
}

int pmfmhd_step_ct_drag(pmfmhd_ctx* c, const pmfmhd_grid* g, const float* const U[9], float* const Unew[9],
                        float* ct_packed, float dt, float drag_impulse, const float target_velocity[3],
                        void* stream) {
  if (c == nullptr || ct_packed == nullptr) return PMFMHD_EINVAL;
  int rc = check_grid(g);
  if (rc) return rc;
  if (!all_periodic(g)) return PMFMHD_EUNSUPPORTED;
  if (!nonnull(U, 9) || !nonnull(Unew, 9)) return PMFMHD_EINVAL;
  if (!std::isfinite(dt)) return PMFMHD_EINVAL;
  if (!std::isfinite(drag_impulse) || !(drag_impulse >= 0.0f)) return PMFMHD_EINVAL;
  SourceTerms st;
  st.src = SRC_DRAG;
  st.drag = drag_coefficients(drag_impulse, target_velocity);
  return enqueue_ct(c, g, U, Unew, ct_packed, dt, nullptr, false, false, as_stream(stream), &st);
}

int pmfmhd_step_radiation(pmfmhd_ctx* c, const pmfmhd_grid* g, const float* const U[9], float* const Unew[9],
                          float* ct_packed, float* correction, float dt, float ch, float decay, float drag_impulse,
                          int flags, void* stream) {
  if (c == nullptr || correction == nullptr) return PMFMHD_EINVAL;
  int rc = check_grid(g);
  if (rc) return rc;
  if (!all_periodic(g)) return PMFMHD_EUNSUPPORTED;
  for (int f = 0; f < 8; ++f)
    if (U[f] == nullptr) return PMFMHD_EINVAL;
  if (!nonnull(Unew, 9)) return PMFMHD_EINVAL;
  if (flags & ~(PMFMHD_RAD_TRACK_DENSITY | PMFMHD_RAD_TRACK_MAGNETIC | PMFMHD_RAD_TRACK_ENERGY |
                PMFMHD_RAD_CHECK_ADMISSIBILITY | PMFMHD_RAD_ROBUST_FALLBACK | PMFMHD_RAD_GLOBAL_FALLBACK |
                PMFMHD_RAD_MASKED_FALLBACK))
    return PMFMHD_EINVAL;
  if (!std::isfinite(dt) || !std::isfinite(drag_impulse) || !(drag_impulse >= 0.0f)) return PMFMHD_EINVAL;
  const bool ct = ct_packed != nullptr;
  // the masked fallback exists in the cube kernel only, which runs GLM states
  if (ct && (flags & PMFMHD_RAD_MASKED_FALLBACK)) return PMFMHD_EUNSUPPORTED;
  if (!ct && (!std::isfinite(ch) || !std::isfinite(decay) || !(ch > 0.0f))) return PMFMHD_EINVAL;
  // fallback steps swap the scheme without touching the caller's recon/riemann choice
  // (integrator_ref.jl:243-246, integrator_cube.jl:524-529)
  pmfmhd_grid g2 = *g;
  int rf = flags & (RAD_TRACK_DENSITY | RAD_TRACK_MAGNETIC | RAD_TRACK_ENERGY | RAD_CHECK);
  if (flags & PMFMHD_RAD_ROBUST_FALLBACK) {
    g2.recon = PMFMHD_RECON_PLM_MINMOD;
    g2.riemann = PMFMHD_RIEMANN_HLL;
  } else if (flags & PMFMHD_RAD_GLOBAL_FALLBACK) {
    g2.riemann = PMFMHD_RIEMANN_LLF;
  }
  // integrator_cube.jl:524-529: the global fallback launches with CHECK == 3, piecewise-constant
  // states and the admissibility test (with the robust solver if both are asked for)
  if (flags & PMFMHD_RAD_GLOBAL_FALLBACK) rf |= RAD_CHECK | RAD_FIRST_ORDER;
  // integrator_cube.jl:527: without the global fallback, `fallback` launches with CHECK == 2, the
  // per-cell mask in slot 4 of the correction buffer and the admissibility test
  const float* mask = nullptr;
  if ((flags & PMFMHD_RAD_MASKED_FALLBACK) && !(flags & PMFMHD_RAD_GLOBAL_FALLBACK)) {
    rf |= RAD_CHECK | RAD_MASKED;
    const long long nc = ncells(g);
    mask = correction + 4 * nc;
    if (flags & PMFMHD_RAD_TRACK_DENSITY) {
      // the density increments are accumulated into that slot by this launch: read the mask
      // from a copy taken before it
      std::lock_guard<std::mutex> lk(c->mu);
      if (c->mask_cells < nc) {
        cudaFree(c->d_mask);
        c->d_mask = nullptr;
        c->mask_cells = 0;
        PMF_CK(cudaMalloc(&c->d_mask, sizeof(float) * nc));
        c->mask_cells = nc;
      }
      PMF_CK(cudaMemcpyAsync(c->d_mask, mask, sizeof(float) * nc, cudaMemcpyDeviceToDevice, as_stream(stream)));
      mask = c->d_mask;
    }
  }
  // psi is read from slot 0 of the correction buffer, as the reference passes the buffer in
  // place of U[9]
  const float* Uin[9];
  for (int f = 0; f < 8; ++f) Uin[f] = U[f];
  Uin[8] = correction;
  SourceTerms st;
  st.src = SRC_RAD;
  st.drag = drag_coefficients(drag_impulse, nullptr);
  st.corr = correction;
  st.rad_flags = rf;
  st.mask = mask;
  if (ct)
    return enqueue_ct(c, &g2, Uin, Unew, ct_packed, dt, nullptr, false, (rf & RAD_TRACK_MAGNETIC) != 0,
                      as_stream(stream), &st);
  return enqueue_glm(c, &g2, Uin, Unew, dt, ch, decay, nullptr, false, as_stream(stream), &st);
}

int pmfmhd_max_wavespeed(pmfmhd_ctx* c, const pmfmhd_grid* g, const float* const U[9], float* smax, void* stream) {
  if (c == nullptr || smax == nullptr) return PMFMHD_EINVAL;
  int rc = check_grid(g);
  if (rc) return rc;
  if (!nonnull(U, 9)) return PMFMHD_EINVAL;
  cudaStream_t s = as_stream(stream);
  CPtr9 u;
  for (int f = 0; f < 9; ++f) u.p[f] = U[f];
  PMF_CK(cudaMemsetAsync(c->d_smax, 0, sizeof(unsigned int), s));
  wavespeed_kernel<<<aux_blocks(c, ncells(g)), AUX_THREADS, 0, s>>>(u, (int)ncells(g), phys_of(g), c->d_smax);
  PMF_CK(cudaGetLastError());
  return read_smax(c, smax, s);
}

int pmfmhd_compute_dt(pmfmhd_ctx* c, const pmfmhd_grid* g, const float* const U[9], float cfl, float* dt,
                      float* smax, void* stream) {
  if (dt == nullptr || !std::isfinite(cfl) || !(cfl > 0.0f)) return PMFMHD_EINVAL;
  float sm;
  int rc = pmfmhd_max_wavespeed(c, g, U, &sm, stream);
  if (rc) return rc;
  const float eps = 1.1920929e-7f;  // eps(Float32)
  *dt = cfl * g->dx / (sm > eps ? sm : eps);  // timestep.jl:39
  if (smax) *smax = sm;
  return PMFMHD_OK;
}

int pmfmhd_last_wavespeed(pmfmhd_ctx* c, float* smax, void* stream) {
  if (c == nullptr || smax == nullptr) return PMFMHD_EINVAL;
  return read_smax(c, smax, as_stream(stream));
}

int pmfmhd_max_divb(pmfmhd_ctx* c, const pmfmhd_grid* g, const float* const U[9], double* out, void* stream) {
  if (c == nullptr || out == nullptr) return PMFMHD_EINVAL;
  int rc = check_grid(g);
  if (rc) return rc;
  if (!nonnull(U, 9)) return PMFMHD_EINVAL;
  cudaStream_t s = as_stream(stream);
  PMF_CK(cudaMemsetAsync(c->d_u64, 0, sizeof(unsigned long long), s));
  divb_kernel<<<aux_blocks(c, ncells(g)), AUX_THREADS, 0, s>>>(U[5], U[6], U[7], g->nx, g->ny, g->nz, g->bc[0],
                                                                g->bc[1], g->bc[2], 1.0 / (2.0 * (double)g->dx),
                                                                c->d_u64);
  PMF_CK(cudaGetLastError());
  PMF_CK(cudaMemcpyAsync(c->h_pin, c->d_u64, 8, cudaMemcpyDeviceToHost, s));
  PMF_CK(cudaStreamSynchronize(s));
  std::memcpy(out, c->h_pin, 8);
  return PMFMHD_OK;
}

int pmfmhd_max_divb_face(pmfmhd_ctx* c, const pmfmhd_grid* g, const float* ct, double* out, void* stream) {
  if (c == nullptr || out == nullptr || ct == nullptr) return PMFMHD_EINVAL;
  int rc = check_grid(g);
  if (rc) return rc;
  cudaStream_t s = as_stream(stream);
  const long long nc = ncells(g);
  PMF_CK(cudaMemsetAsync(c->d_u64, 0, sizeof(unsigned long long), s));
  divb_face_kernel<<<aux_blocks(c, nc), AUX_THREADS, 0, s>>>(ct, ct + nc, ct + 2 * nc, g->nx, g->ny, g->nz,
                                                              1.0 / (double)g->dx, c->d_u64);
  PMF_CK(cudaGetLastError());
  PMF_CK(cudaMemcpyAsync(c->h_pin, c->d_u64, 8, cudaMemcpyDeviceToHost, s));
  PMF_CK(cudaStreamSynchronize(s));
  std::memcpy(out, c->h_pin, 8);
  return PMFMHD_OK;
}

int pmfmhd_conserved_totals(pmfmhd_ctx* c, const pmfmhd_grid* g, const float* const U[9], double out[8],
                            void* stream) {
  if (c == nullptr || out == nullptr) return PMFMHD_EINVAL;
  int rc = check_grid(g);
  if (rc) return rc;
  if (!nonnull(U, 9)) return PMFMHD_EINVAL;
  cudaStream_t s = as_stream(stream);
  CPtr9 u;
  for (int f = 0; f < 9; ++f) u.p[f] = U[f];
  const int nb = std::min(aux_blocks(c, ncells(g)), kTotBlocksMax);
  totals_partial_kernel<<<nb, AUX_THREADS, 0, s>>>(u, (int)ncells(g), c->d_partial);
  const float dV = g->dx * g->dx * g->dx;  // s.dx^3 in T (diagnostics.jl:45)
  totals_final_kernel<<<1, 32, 0, s>>>(c->d_partial, nb, (double)dV, c->d_tot);
  PMF_CK(cudaGetLastError());
  PMF_CK(cudaMemcpyAsync(c->h_pin, c->d_tot, 64, cudaMemcpyDeviceToHost, s));
  PMF_CK(cudaStreamSynchronize(s));
  std::memcpy(out, c->h_pin, 64);
  return PMFMHD_OK;
}

int pmfmhd_ct_faces_from_potential(pmfmhd_ctx* c, const pmfmhd_grid* g, const float* const A[3], float* const U[9],
                                   float* ct, void* stream) {
  if (c == nullptr || ct == nullptr) return PMFMHD_EINVAL;
  int rc = check_grid(g);
  if (rc) return rc;
  if (!all_periodic(g)) return PMFMHD_EUNSUPPORTED;
  if (!nonnull(A, 3) || !nonnull(U, 9)) return PMFMHD_EINVAL;
  cudaStream_t s = as_stream(stream);
  const int nb = aux_blocks(c, ncells(g));
  ct_curl_kernel<<<nb, AUX_THREADS, 0, s>>>(A[0], A[1], A[2], ct, g->nx, g->ny, g->nz, 1.0f / g->dx);
  PMF_CK(cudaGetLastError());
  return pmfmhd_ct_install_faces(c, g, U, ct, stream);
}

int pmfmhd_ct_install_faces(pmfmhd_ctx* c, const pmfmhd_grid* g, float* const U[9], float* ct, void* stream) {
  if (c == nullptr || ct == nullptr) return PMFMHD_EINVAL;
  int rc = check_grid(g);
  if (rc) return rc;
  if (!all_periodic(g)) return PMFMHD_EUNSUPPORTED;
  if (!nonnull(U, 9)) return PMFMHD_EINVAL;
  cudaStream_t s = as_stream(stream);
  const long long nc = ncells(g);
  PMF_CK(cudaMemsetAsync(ct + (size_t)CT_RBX * nc, 0, sizeof(float) * 3 * (size_t)nc, s));
  MPtr9 u;
  for (int f = 0; f < 9; ++f) u.p[f] = U[f];
  ct_cell_from_faces_kernel<<<aux_blocks(c, nc), AUX_THREADS, 0, s>>>(ct, u, g->nx, g->ny, g->nz);
  PMF_CK(cudaGetLastError());
  return PMFMHD_OK;
}

int pmfmhd_run_glm(pmfmhd_ctx* c, const pmfmhd_grid* g, float* const U[9], float* const scratch[9], int nsteps,
                   float dt, float ch, float decay, float* const resid[7], void* stream) {
  if (c == nullptr || nsteps < 0) return PMFMHD_EINVAL;
  int rc = check_grid(g);
  if (rc) return rc;
  if (!nonnull(U, 9) || !nonnull(scratch, 9)) return PMFMHD_EINVAL;
  if (!std::isfinite(dt) || !std::isfinite(ch) || !std::isfinite(decay) || !(ch > 0.0f)) return PMFMHD_EINVAL;
  bool comp;
  if ((rc = resid_mode(resid, &comp))) return rc;
  if (nsteps == 0) return PMFMHD_OK;
  const Tune t = tune_for(c, g, false, comp);
  // graph key: every input that changes the recorded launches
  std::vector<unsigned char> key(sizeof(pmfmhd_grid) + 25 * sizeof(void*) + 3 * sizeof(float) + 3 * sizeof(int));
  unsigned char* k = key.data();
  std::memcpy(k, g, sizeof(pmfmhd_grid)); k += sizeof(pmfmhd_grid);
  std::memcpy(k, U, 9 * sizeof(void*)); k += 9 * sizeof(void*);
  std::memcpy(k, scratch, 9 * sizeof(void*)); k += 9 * sizeof(void*);
  for (int i = 0; i < 7; ++i) {
    void* p = comp ? (void*)resid[i] : nullptr;
    std::memcpy(k, &p, sizeof(void*)); k += sizeof(void*);
  }
  std::memcpy(k, &dt, 4); k += 4;
  std::memcpy(k, &ch, 4); k += 4;
  std::memcpy(k, &decay, 4); k += 4;
  std::memcpy(k, &nsteps, 4); k += 4;
  std::memcpy(k, &t.ty, 4); k += 4;
  std::memcpy(k, &t.tz, 4); k += 4;
  cudaStream_t s = as_stream(stream);
  std::lock_guard<std::mutex> lk(c->mu);
  for (auto& e : c->graphs) {
    if (e.key == key) {
      PMF_CK(cudaGraphLaunch(e.exec, s));
      return PMFMHD_OK;
    }
  }
  // Record nsteps ping-pong steps on the capture stream, then replay on the caller's stream.
  PMF_CK(cudaStreamBeginCapture(c->cap, cudaStreamCaptureModeThreadLocal));
  const float dtdx = dt / g->dx;
  for (int n = 0; n < nsteps; ++n) {
    float* const* src = (n % 2 == 0) ? U : scratch;
    float* const* dst = (n % 2 == 0) ? scratch : U;
    StepArgs a;
    fill_glm_args(a, src, dst, resid, comp, dtdx, ch, decay, c->d_smax);
    cudaMemsetAsync(c->d_smax, 0, sizeof(unsigned int), c->cap);
    int lrc = launch_step(c, g, a, t, false, comp, c->cap);
    if (lrc != PMFMHD_OK) {
      cudaGraph_t dead = nullptr;
      cudaStreamEndCapture(c->cap, &dead);
      if (dead) cudaGraphDestroy(dead);
      cudaGetLastError();  // leave no error from the abandoned capture behind
      return lrc;
    }
  }
  cudaGraph_t graph;
  PMF_CK(cudaStreamEndCapture(c->cap, &graph));
  cudaGraphExec_t exec;
  cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    last_cuda_error() = std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e);
    return PMFMHD_ECUDA;
  }
  if (c->graphs.size() >= 16) {
    cudaGraphExecDestroy(c->graphs.front().exec);
    c->graphs.erase(c->graphs.begin());
  }
  c->graphs.push_back(GraphEntry{key, exec});
  PMF_CK(cudaGraphLaunch(exec, s));
  return PMFMHD_OK;
}

int pmfmhd_autotune(pmfmhd_ctx* c, const pmfmhd_grid* g, const float* const U[9], int mhd_solver, int compensated,
                    void* stream) {
  if (c == nullptr) return PMFMHD_EINVAL;
  int rc = check_grid(g);
  if (rc) return rc;
  if (!nonnull(U, 9)) return PMFMHD_EINVAL;
  const bool ct = mhd_solver == 1;
  if (ct && !all_periodic(g)) return PMFMHD_EUNSUPPORTED;
  const bool comp = compensated != 0;
  cudaStream_t s = as_stream(stream);
  const long long nc = ncells(g);
  // scratch copies so the caller's state is never touched
  const size_t nfl = (size_t)nc * (9 + 9 + 7 + (ct ? CT_NSLOT : 0));
  float* buf = nullptr;
  if (cudaMalloc(&buf, nfl * sizeof(float)) != cudaSuccess) return PMFMHD_ENOMEM;
  float* in[9];
  float* outp[9];
  float* res[7];
  for (int f = 0; f < 9; ++f) { in[f] = buf + (size_t)f * nc; outp[f] = buf + (size_t)(9 + f) * nc; }
  for (int i = 0; i < 7; ++i) res[i] = buf + (size_t)(18 + i) * nc;
  float* ctp = ct ? buf + (size_t)25 * nc : nullptr;
  int result = PMFMHD_OK;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  for (int f = 0; f < 9 && result == PMFMHD_OK; ++f)
    if (cudaMemcpyAsync(in[f], U[f], nc * sizeof(float), cudaMemcpyDeviceToDevice, s) != cudaSuccess)
      result = PMFMHD_ECUDA;
  cudaMemsetAsync(res[0], 0, (size_t)7 * nc * sizeof(float), s);
  if (ct) cudaMemsetAsync(ctp, 0, (size_t)CT_NSLOT * nc * sizeof(float), s);
  Tune best = default_tune(c, g);
  float best_ms = 1e30f;
  std::vector<int> tzs = {8, 32};
  for (int ty : kTileRows) {
    if (ty > 5 && g->ny < ty) continue;
    for (int tz : tzs) {
      Tune t{ty, tz};
      float ms_sum = 0.0f;
      for (int rep = 0; rep < 4 && result == PMFMHD_OK; ++rep) {
        StepArgs a;
        fill_glm_args(a, in, outp, res, comp, 1e-4f / g->dx, 1.0f, 1.0f, c->d_smax);
        if (ct) {
          for (int d = 0; d < 3; ++d) a.face[d] = ctp + (size_t)d * nc;
          for (int k = 0; k < CT_NWORK; ++k) a.work[k] = ctp + (size_t)(CT_MFX + k) * nc;
          a.smax_bits = nullptr;
        }
        cudaEventRecord(e0, s);
        int lrc = launch_step(c, g, a, t, ct, comp, s);
        cudaEventRecord(e1, s);
        if (lrc != PMFMHD_OK) { result = lrc; break; }
        if (cudaEventSynchronize(e1) != cudaSuccess) { result = PMFMHD_ECUDA; break; }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0) ms_sum += ms;  // first launch is a warm-up
      }
      if (result != PMFMHD_OK) break;
      if (ms_sum < best_ms) { best_ms = ms_sum; best = t; }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamSynchronize(s);
  cudaFree(buf);
  if (result == PMFMHD_OK) {
    std::lock_guard<std::mutex> lk(c->mu);
    c->tune[TuneKey{g->nx, g->ny, g->nz, ct, comp, g->recon, g->riemann}] = best;
  }
  return result;
}

int pmfmhd_step_glm_census(pmfmhd_ctx* c, const pmfmhd_grid* g, const float* const U[9], float* const Unew[9],
                           float dt, float ch, float decay, uint64_t out[3], void* stream) {
  if (c == nullptr || out == nullptr) return PMFMHD_EINVAL;
  int rc = check_grid(g);
  if (rc) return rc;
  if (!nonnull(U, 9) || !nonnull(Unew, 9)) return PMFMHD_EINVAL;
  if (!std::isfinite(dt) || !std::isfinite(ch) || !std::isfinite(decay) || !(ch > 0.0f)) return PMFMHD_EINVAL;
  if (g->recon != PMFMHD_RECON_PLM || g->riemann != PMFMHD_RIEMANN_HLLD) return PMFMHD_EUNSUPPORTED;
  cudaStream_t s = as_stream(stream);
  unsigned long long* cnt = c->d_u64 + 8;  // 64 bytes past the FP64-max cell
  PMF_CK(cudaMemsetAsync(cnt, 0, 3 * sizeof(unsigned long long), s));
  StepArgs a;
  fill_glm_args(a, U, Unew, nullptr, false, dt / g->dx, ch, decay, c->d_smax);
  a.census = cnt;
  PMF_CK(cudaMemsetAsync(c->d_smax, 0, sizeof(unsigned int), s));
  Tune t = tune_for(c, g, false, false);
  t.ty = kCensusRows;
  const StepKernelInfo k = step_census_kernel_info();
  if ((rc = launch_step(c, g, a, t, false, false, s, SRC_NONE, &k))) return rc;
  PMF_CK(cudaMemcpyAsync(c->h_pin, cnt, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
  PMF_CK(cudaStreamSynchronize(s));
  unsigned long long v[3];
  std::memcpy(v, c->h_pin, sizeof(v));
  for (int q = 0; q < 3; ++q) out[q] = (uint64_t)v[q];
  return PMFMHD_OK;
}

int pmfmhd_set_tma_stall(pmfmhd_ctx* c, int polls) {
  if (c == nullptr || polls < 0) return PMFMHD_EINVAL;
  std::lock_guard<std::mutex> lk(c->mu);
  c->tma_stall_polls = polls;
  return PMFMHD_OK;
}

int pmfmhd_status(pmfmhd_ctx* c, int clear, void* stream) {
  if (c == nullptr) return PMFMHD_EINVAL;
  cudaStream_t s = as_stream(stream);
  PMF_CK(cudaMemcpyAsync(c->h_pin, c->d_status, sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
  PMF_CK(cudaStreamSynchronize(s));
  unsigned int bits;
  std::memcpy(&bits, c->h_pin, sizeof(bits));
  if (clear) PMF_CK(cudaMemsetAsync(c->d_status, 0, sizeof(unsigned int), s));
  return bits & 1u ? PMFMHD_ETIMEOUT : PMFMHD_OK;
}

int pmfmhd_set_tile(pmfmhd_ctx* c, const pmfmhd_grid* g, int mhd_solver, int compensated, int rows, int planes) {
  if (c == nullptr) return PMFMHD_EINVAL;
  int rc = check_grid(g);
  if (rc) return rc;
  bool known = false;
  for (int ty : kTileRows) known |= ty == rows;
  if (!known || planes < 1) return PMFMHD_EINVAL;
  std::lock_guard<std::mutex> lk(c->mu);
  c->tune[TuneKey{g->nx, g->ny, g->nz, mhd_solver == 1, compensated != 0, g->recon, g->riemann}] =
      Tune{rows, std::min(planes, g->nz)};
  return PMFMHD_OK;
}

int pmfmhd_get_tile(pmfmhd_ctx* c, const pmfmhd_grid* g, int mhd_solver, int compensated, int* rows, int* planes) {
  if (c == nullptr || rows == nullptr || planes == nullptr) return PMFMHD_EINVAL;
  int rc = check_grid(g);
  if (rc) return rc;
  const Tune t = tune_for(c, g, mhd_solver == 1, compensated != 0);
  *rows = t.ty;
  *planes = t.tz;
  return PMFMHD_OK;
}

}  // extern "C"
