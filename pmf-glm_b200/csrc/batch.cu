// Batched driver: many independent boxes of uneven sizes advanced together.
//
// One step of the batch is, with every pointer static (so it is recorded once per buffer
// parity as a CUDA graph and replayed):
//   1. per (solver family, tile height) one persistent launch of mhd_batch_kernel, which
//      splits the concatenated (column, plane) spaces of its boxes evenly over the CTAs;
//      each box reads its own {dt/dx, ch, decay} from device memory and reduces the max
//      signal speed of its new state into its own slot;
//   2. for constrained-transport boxes, the EMF / face / cell-B column kernels over all CT
//      boxes (each block one 32 x 8 x 16 column tile of one box, so each block reduces one
//      box's signal speed);
//   3. one thread per box turns its signal speed into the next step's dt, ch and decay the
//      way `evolve!` does (driver.jl:48-71, timestep.jl:37-41) and advances its clock.
// Nothing returns to the host between steps.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <vector>

#include "aux_kernels.cuh"
#include "host_internal.h"
#include "step_kernel.cuh"

using namespace pmf;
using namespace pmf::host;

namespace {

struct BoxMeta {
  float cfl, ch_fac, cr, dx;
  int ct;
};

// One CT box seen by the batched companion kernels.
struct CtView {
  float* ct;
  MPtr9 Un;
  int nx, ny, nz;
  int block0;           // first block of this box
  const float* dscal;   // {dt/dx, ch, decay, dt}
  unsigned int* smax_bits;
  Phys P;
  int comp_faces;
};

__device__ __forceinline__ int find_view(const CtView* v, int n, int blk) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (v[mid].block0 <= blk) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// The block's column tile of its box: blocks block0.. of a box enumerate its (tx, ty, tz)
// tiles of the column kernels, x fastest.
__device__ __forceinline__ void col_tile(const CtView& b, int blk, int& tx, int& ty, int& tz) {
  const int ntx = (b.nx + CTC_X - 1) / CTC_X, nty = (b.ny + CTC_Y - 1) / CTC_Y;
  const int l = blk - b.block0;
  tx = l % ntx;
  ty = (l / ntx) % nty;
  tz = l / (ntx * nty);
}

__device__ __forceinline__ float* ct_slot(const CtView& b, int k) {
  return b.ct + (size_t)k * ((size_t)b.nx * b.ny * b.nz);
}

__global__ void __launch_bounds__(AUX_THREADS) batch_ct_emf_kernel(const CtView* __restrict__ v, int n) {
  const CtView& b = v[find_view(v, n, blockIdx.x)];
  int tx, ty, tz;
  col_tile(b, blockIdx.x, tx, ty, tz);
  ct_emf_col(ct_slot(b, CT_MFX), ct_slot(b, CT_MFY), ct_slot(b, CT_MFZ), ct_slot(b, CT_FXBY), ct_slot(b, CT_FXBZ),
             ct_slot(b, CT_FYBX), ct_slot(b, CT_FYBZ), ct_slot(b, CT_FZBX), ct_slot(b, CT_FZBY), ct_slot(b, CT_ECX),
             ct_slot(b, CT_ECY), ct_slot(b, CT_ECZ), ct_slot(b, CT_EX), ct_slot(b, CT_EY), ct_slot(b, CT_EZ), b.nx,
             b.ny, b.nz, tx, ty, tz);
}

__global__ void __launch_bounds__(AUX_THREADS) batch_ct_face_kernel(const CtView* __restrict__ v, int n) {
  const CtView& b = v[find_view(v, n, blockIdx.x)];
  int tx, ty, tz;
  col_tile(b, blockIdx.x, tx, ty, tz);
  const float dtdx = b.dscal[0];
  if (b.comp_faces)
    ct_face_col<true>(ct_slot(b, CT_EX), ct_slot(b, CT_EY), ct_slot(b, CT_EZ), ct_slot(b, CT_BXF), ct_slot(b, CT_BYF),
                      ct_slot(b, CT_BZF), ct_slot(b, CT_RBX), ct_slot(b, CT_RBY), ct_slot(b, CT_RBZ), b.nx, b.ny,
                      b.nz, dtdx, tx, ty, tz);
  else
    ct_face_col<false>(ct_slot(b, CT_EX), ct_slot(b, CT_EY), ct_slot(b, CT_EZ), ct_slot(b, CT_BXF),
                       ct_slot(b, CT_BYF), ct_slot(b, CT_BZF), ct_slot(b, CT_RBX), ct_slot(b, CT_RBY),
                       ct_slot(b, CT_RBZ), b.nx, b.ny, b.nz, dtdx, tx, ty, tz);
}

__global__ void __launch_bounds__(AUX_THREADS) batch_ct_bcc_kernel(const CtView* __restrict__ v, int n) {
  const CtView& b = v[find_view(v, n, blockIdx.x)];
  int tx, ty, tz;
  col_tile(b, blockIdx.x, tx, ty, tz);
  float m = ct_bcc_col(ct_slot(b, CT_BXF), ct_slot(b, CT_BYF), ct_slot(b, CT_BZF), b.Un, b.nx, b.ny, b.nz, b.P, true,
                       tx, ty, tz);
  m = block_reduce_max(m);
  if (threadIdx.x == 0) atomicMax(b.smax_bits, __float_as_uint(m));
}

// Per-box CFL: the next dt, ch and decay from the signal speed of the current state.
// `account` adds the step just taken to the box's clock.
__global__ void batch_dt_kernel(const BoxMeta* __restrict__ meta, float* dscal, double* dtf_out,
                                unsigned int* smax_bits, double* t, int nbox, int account) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbox) return;
  if (account) t[b] += dtf_out[b];
  const BoxMeta m = meta[b];
  const float smax = __uint_as_float(smax_bits[b]);
  smax_bits[b] = 0u;
  const float eps = 1.1920929e-7f;                       // eps(Float32)
  const float dt = __fdiv_rn(m.cfl * m.dx, fmaxf(smax, eps));  // timestep.jl:39
  double dtf;
  float ch, decay;
  if (m.ct) {
    ch = 0.0f;
    dtf = (double)dt;
    decay = 1.0f;
  } else {
    ch = m.ch_fac * smax;                                            // driver.jl:59
    dtf = (double)dt * (double)smax / (double)fmaxf(smax, ch);       // driver.jl:60
    const float a = __fdiv_rn(-m.cr * ch * (float)dtf, m.dx);         // driver.jl:29, in T
    decay = (float)exp((double)a);                                   // the exponential in FP64
  }
  dscal[4 * b + 0] = __fdiv_rn((float)dtf, m.dx);
  dscal[4 * b + 1] = ch;
  dscal[4 * b + 2] = decay;
  dscal[4 * b + 3] = (float)dtf;
  dtf_out[b] = dtf;
}

struct Group {
  bool ct, comp;
  int recon, rsol, ty;
  std::vector<int> ids;
  BoxStep* d_desc[2] = {nullptr, nullptr};
  long long Q = 0;
  int blocks = 0;
  StepKernelInfo info{};
  BatchKernel fn = nullptr;
};

}  // namespace

struct pmfmhd_batch {
  pmfmhd_ctx* ctx = nullptr;
  std::vector<pmfmhd_box> boxes;
  std::vector<Group> groups;
  float* d_dscal = nullptr;
  double* d_dtf = nullptr;
  double* d_t = nullptr;
  unsigned int* d_smax = nullptr;
  BoxMeta* d_meta = nullptr;
  CtView* d_ct[2] = {nullptr, nullptr};
  int nct = 0, ct_blocks = 0;
  int parity = 0;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  cudaStream_t last = nullptr;
};

namespace {

void free_batch(pmfmhd_batch* b) {
  if (b == nullptr) return;
  for (int p = 0; p < 2; ++p) {
    if (b->graph[p]) cudaGraphExecDestroy(b->graph[p]);
    cudaFree(b->d_ct[p]);
    for (auto& g : b->groups) cudaFree(g.d_desc[p]);
  }
  cudaFree(b->d_dscal);
  cudaFree(b->d_dtf);
  cudaFree(b->d_t);
  cudaFree(b->d_smax);
  cudaFree(b->d_meta);
  delete b;
}

// Enqueue one step of the batch for buffer parity p on stream s.
int enqueue_batch_step(pmfmhd_batch* b, int p, cudaStream_t s) {
  for (auto& g : b->groups) {
    if (g.Q == 0) continue;
    int n = (int)g.ids.size();
    void* args[] = {(void*)&g.d_desc[p], (void*)&n, (void*)&g.Q};
    PMF_CK(cudaLaunchKernel((const void*)g.fn, dim3(g.blocks), dim3(g.info.threads), args, g.info.smem_bytes, s));
  }
  if (b->nct > 0) {
    batch_ct_emf_kernel<<<b->ct_blocks, AUX_THREADS, 0, s>>>(b->d_ct[p], b->nct);
    batch_ct_face_kernel<<<b->ct_blocks, AUX_THREADS, 0, s>>>(b->d_ct[p], b->nct);
    batch_ct_bcc_kernel<<<b->ct_blocks, AUX_THREADS, 0, s>>>(b->d_ct[p], b->nct);
  }
  const int nbox = (int)b->boxes.size();
  batch_dt_kernel<<<(nbox + 127) / 128, 128, 0, s>>>(b->d_meta, b->d_dscal, b->d_dtf, b->d_smax, b->d_t, nbox, 1);
  PMF_CK(cudaGetLastError());
  return PMFMHD_OK;
}

}  // namespace

extern "C" {

int pmfmhd_batch_create(pmfmhd_ctx* c, const pmfmhd_box* boxes, int nbox, pmfmhd_batch** out) {
  if (out) *out = nullptr;
  if (c == nullptr || boxes == nullptr || nbox < 1 || out == nullptr) return PMFMHD_EINVAL;
  for (int i = 0; i < nbox; ++i) {
    const pmfmhd_box& x = boxes[i];
    int rc = check_grid(&x.grid);
    if (rc) return rc;
    for (int f = 0; f < 9; ++f)
      if (x.U[f] == nullptr || x.scratch[f] == nullptr) return PMFMHD_EINVAL;
    int nres = 0;
    for (int r = 0; r < 7; ++r) nres += x.resid[r] != nullptr;
    if (nres != 0 && nres != 7) return PMFMHD_EINVAL;
    if (x.mhd_solver != 0 && x.mhd_solver != 1) return PMFMHD_EINVAL;
    if (x.mhd_solver == 1 && (x.ct_packed == nullptr || !all_periodic(&x.grid))) return PMFMHD_EUNSUPPORTED;
    if (!(x.cfl > 0.0f) || !(x.glm_ch_fac > 0.0f) || !(x.glm_cr >= 0.0f)) return PMFMHD_EINVAL;
  }
  PMF_CK(cudaSetDevice(c->device));
  pmfmhd_batch* b = new pmfmhd_batch();
  b->ctx = c;
  b->boxes.assign(boxes, boxes + nbox);
  auto fail = [&](int rc) {
    free_batch(b);
    return rc;
  };
  if (cudaMalloc(&b->d_dscal, sizeof(float) * 4 * nbox) != cudaSuccess ||
      cudaMalloc(&b->d_dtf, sizeof(double) * nbox) != cudaSuccess ||
      cudaMalloc(&b->d_t, sizeof(double) * nbox) != cudaSuccess ||
      cudaMalloc(&b->d_smax, sizeof(unsigned int) * nbox) != cudaSuccess ||
      cudaMalloc(&b->d_meta, sizeof(BoxMeta) * nbox) != cudaSuccess)
    return fail(PMFMHD_ENOMEM);
  // Groups by (solver, compensation, reconstruction, Riemann solver). One tile height per
  // group, the one tuned for the group's largest box: the single-box tuning of a small box
  // favours short tiles (more CTAs for a box that cannot fill the GPU alone), but in a batch
  // every box shares the persistent CTAs, so the taller tile's lower halo overhead wins and
  // the step stays one launch per group.
  std::map<std::tuple<int, int, int, int>, int> family_ty;
  {
    std::map<std::tuple<int, int, int, int>, long long> family_cells;
    for (int i = 0; i < nbox; ++i) {
      const pmfmhd_box& x = boxes[i];
      const bool ct = x.mhd_solver == 1, comp = x.resid[0] != nullptr;
      const auto fam = std::make_tuple((int)ct, (int)comp, x.grid.recon, x.grid.riemann);
      const long long nc = ncells(&x.grid);
      if (nc > family_cells[fam]) {
        family_cells[fam] = nc;
        family_ty[fam] = tune_for(c, &x.grid, ct, comp).ty;
      }
    }
  }
  std::map<std::tuple<int, int, int, int, int>, int> gidx;
  std::vector<BoxMeta> meta(nbox);
  for (int i = 0; i < nbox; ++i) {
    const pmfmhd_box& x = boxes[i];
    const bool ct = x.mhd_solver == 1, comp = x.resid[0] != nullptr;
    Tune t = tune_for(c, &x.grid, ct, comp);
    t.ty = family_ty[std::make_tuple((int)ct, (int)comp, x.grid.recon, x.grid.riemann)];
    auto key = std::make_tuple((int)ct, (int)comp, x.grid.recon, x.grid.riemann, t.ty);
    if (!gidx.count(key)) {
      Group g;
      g.ct = ct; g.comp = comp; g.recon = x.grid.recon; g.rsol = x.grid.riemann; g.ty = t.ty;
      g.info = step_kernel_info(t.ty, g.recon, g.rsol, ct, comp);
      g.fn = batch_kernel(t.ty, g.recon, g.rsol, ct, comp);
      if (g.info.fn == nullptr || g.fn == nullptr) return fail(PMFMHD_EUNSUPPORTED);
      gidx[key] = (int)b->groups.size();
      b->groups.push_back(g);
    }
    b->groups[gidx[key]].ids.push_back(i);
    meta[i] = BoxMeta{x.cfl, x.glm_ch_fac, x.glm_cr, x.grid.dx, (int)ct};
  }
  // per-group descriptors for both buffer parities
  for (auto& g : b->groups) {
    // largest boxes first, so that CTAs covering small boxes do not trail
    std::stable_sort(g.ids.begin(), g.ids.end(), [&](int a_, int b_) {
      return ncells(&boxes[a_].grid) > ncells(&boxes[b_].grid);
    });
    std::vector<BoxStep> desc[2];
    long long q = 0;
    for (int i : g.ids) {
      const pmfmhd_box& x = boxes[i];
      const long long nc = ncells(&x.grid);
      for (int p = 0; p < 2; ++p) {
        BoxStep d;
        std::memset(&d, 0, sizeof(d));
        StepArgs& a = d.a;
        for (int f = 0; f < 9; ++f) {
          a.U[f] = p == 0 ? x.U[f] : x.scratch[f];
          a.Un[f] = p == 0 ? x.scratch[f] : x.U[f];
        }
        if (g.comp)
          for (int r = 0; r < 7; ++r) a.resid[r] = x.resid[r];
        if (g.ct) {
          for (int k = 0; k < 3; ++k) a.face[k] = x.ct_packed + (size_t)(CT_BXF + k) * nc;
          for (int k = 0; k < CT_NWORK; ++k) a.work[k] = x.ct_packed + (size_t)(CT_MFX + k) * nc;
        }
        a.nx = x.grid.nx; a.ny = x.grid.ny; a.nz = x.grid.nz;
        for (int k = 0; k < 3; ++k) a.bc[k] = x.grid.bc[k];
        a.ntx = (x.grid.nx + TILE_X - 1) / TILE_X;
        a.nty = (x.grid.ny + g.ty - 1) / g.ty;
        a.P = phys_of(&x.grid);
        a.smax_bits = g.ct ? nullptr : b->d_smax + i;
        a.dscal = b->d_dscal + 4 * i;
        a.status = c->d_status;
        a.use_tma = 0;  // the batched kernel stages every plane by cp.async
        d.q0 = q;
        desc[p].push_back(d);
      }
      q += (long long)((x.grid.nx + TILE_X - 1) / TILE_X) * ((x.grid.ny + g.ty - 1) / g.ty) * x.grid.nz;
    }
    g.Q = q;
    if (cudaFuncSetAttribute((const void*)g.fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)g.info.smem_bytes) != cudaSuccess)
      return fail(PMFMHD_ECUDA);
    const int occ = occupancy_of(g.info);
    g.blocks = (int)std::min<long long>((long long)c->sms * occ, std::max<long long>(1, (q + 15) / 16));
    for (int p = 0; p < 2; ++p) {
      if (cudaMalloc(&g.d_desc[p], sizeof(BoxStep) * desc[p].size()) != cudaSuccess) return fail(PMFMHD_ENOMEM);
      if (cudaMemcpy(g.d_desc[p], desc[p].data(), sizeof(BoxStep) * desc[p].size(), cudaMemcpyHostToDevice) !=
          cudaSuccess)
        return fail(PMFMHD_ECUDA);
    }
  }
  // CT companion views
  std::vector<CtView> views[2];
  int blk = 0;
  for (int i = 0; i < nbox; ++i) {
    const pmfmhd_box& x = boxes[i];
    if (x.mhd_solver != 1) continue;
    for (int p = 0; p < 2; ++p) {
      CtView v;
      v.ct = x.ct_packed;
      for (int f = 0; f < 9; ++f) v.Un.p[f] = p == 0 ? x.scratch[f] : x.U[f];
      v.nx = x.grid.nx; v.ny = x.grid.ny; v.nz = x.grid.nz;
      v.block0 = blk;
      v.dscal = b->d_dscal + 4 * i;
      v.smax_bits = b->d_smax + i;
      v.P = phys_of(&x.grid);
      v.comp_faces = x.resid[0] != nullptr;
      views[p].push_back(v);
    }
    const dim3 tiles = ctc_grid(x.grid.nx, x.grid.ny, x.grid.nz);  // column tiles of this box
    blk += (int)(tiles.x * tiles.y * tiles.z);
  }
  b->nct = (int)views[0].size();
  b->ct_blocks = blk;
  if (b->nct > 0)
    for (int p = 0; p < 2; ++p) {
      if (cudaMalloc(&b->d_ct[p], sizeof(CtView) * b->nct) != cudaSuccess) return fail(PMFMHD_ENOMEM);
      if (cudaMemcpy(b->d_ct[p], views[p].data(), sizeof(CtView) * b->nct, cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(PMFMHD_ECUDA);
    }
  // initial signal speeds (timestep.jl) and the first dt of every box
  std::vector<unsigned int> sm(nbox);
  for (int i = 0; i < nbox; ++i) {
    float v;
    int rc = pmfmhd_max_wavespeed(c, &boxes[i].grid, (const float* const*)boxes[i].U, &v, nullptr);
    if (rc) return fail(rc);
    std::memcpy(&sm[i], &v, 4);
  }
  if (cudaMemcpy(b->d_smax, sm.data(), 4 * nbox, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(b->d_meta, meta.data(), sizeof(BoxMeta) * nbox, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(b->d_t, 0, sizeof(double) * nbox) != cudaSuccess ||
      cudaMemset(b->d_dtf, 0, sizeof(double) * nbox) != cudaSuccess)
    return fail(PMFMHD_ECUDA);
  batch_dt_kernel<<<(nbox + 127) / 128, 128>>>(b->d_meta, b->d_dscal, b->d_dtf, b->d_smax, b->d_t, nbox, 0);
  if (cudaDeviceSynchronize() != cudaSuccess) return fail(PMFMHD_ECUDA);
  *out = b;
  return PMFMHD_OK;
}

int pmfmhd_batch_step(pmfmhd_batch* b, int nsteps, void* stream) {
  if (b == nullptr || nsteps < 0) return PMFMHD_EINVAL;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  pmfmhd_ctx* c = b->ctx;
  for (int n = 0; n < nsteps; ++n) {
    const int p = b->parity;
    if (b->graph[p] == nullptr) {
      std::lock_guard<std::mutex> lk(c->mu);
      PMF_CK(cudaStreamBeginCapture(c->cap, cudaStreamCaptureModeThreadLocal));
      int rc = enqueue_batch_step(b, p, c->cap);
      cudaGraph_t graph = nullptr;
      cudaError_t e = cudaStreamEndCapture(c->cap, &graph);
      if (rc != PMFMHD_OK || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();  // leave no error from the abandoned capture behind
        return rc != PMFMHD_OK ? rc : PMFMHD_ECUDA;
      }
      e = cudaGraphInstantiate(&b->graph[p], graph, 0);
      cudaGraphDestroy(graph);
      if (e != cudaSuccess) {
        last_cuda_error() = std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e);
        b->graph[p] = nullptr;
        return PMFMHD_ECUDA;
      }
    }
    PMF_CK(cudaGraphLaunch(b->graph[p], s));
    b->parity ^= 1;
  }
  b->last = s;
  return PMFMHD_OK;
}

int pmfmhd_batch_query(pmfmhd_batch* b, double* t, int32_t* parity, float* dt) {
  if (b == nullptr) return PMFMHD_EINVAL;
  PMF_CK(cudaStreamSynchronize(b->last));
  const int n = (int)b->boxes.size();
  if (t) PMF_CK(cudaMemcpy(t, b->d_t, sizeof(double) * n, cudaMemcpyDeviceToHost));
  if (parity)
    for (int i = 0; i < n; ++i) parity[i] = b->parity;
  if (dt) {
    std::vector<float> ds(4 * n);
    PMF_CK(cudaMemcpy(ds.data(), b->d_dscal, sizeof(float) * 4 * n, cudaMemcpyDeviceToHost));
    for (int i = 0; i < n; ++i) dt[i] = ds[4 * i + 3];
  }
  return PMFMHD_OK;
}

int pmfmhd_batch_destroy(pmfmhd_batch* b) {
  if (b == nullptr) return PMFMHD_OK;
  cudaSetDevice(b->ctx->device);
  cudaDeviceSynchronize();
  free_batch(b);
  return PMFMHD_OK;
}

}  // extern "C"
