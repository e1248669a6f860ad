// Fused MUSCL-Hancock Godunov step (GLM or CT Godunov stage) for sm_100a.
//
// Scheme: the reference's per-cell body (lib/MHDKernels/src/integrator_ref.jl:69-160, shared
// with the shared-memory cube, integrator_cube.jl:295-444): MC-PLM/PPM/minmod offsets, the
// multidimensional Hancock half step, one Riemann problem per face, and
//   U' = U + dt/dx * (((Fxl-Fxh) + (Fyl-Fyh)) + (Fzl-Fzh)),  psi' *= decay.
//
// Decomposition (B200-specific, not the reference's 4^3 cube): one CTA owns a column of
// 32 x TY cells in (x, y) and streams through a range of z-planes one plane at a time.
//   * row warps w = 0..TY+1 <-> rows y0+w-1 (w = 0 and TY+1 are the y-halo rows); lane l
//     <-> column x0+l. One more "halo warp" computes, per owned row, the two x-halo cells
//     x0-1 and x0+32. Every thread computes the Hancock state of its cell once per plane.
//   * x-faces are solved in registers: lane l solves the face below its cell with the left
//     state from lane l-1 by __shfl_up (lane 0 takes the left halo cell's state from shared
//     memory); the face above lane 31 is solved by the halo warp.
//   * y-faces exchange one 9-float state per thread through shared memory.
//   * z-faces never leave the column: each thread keeps the upper z-face state, the lower
//     z-face flux and the x/y flux divergence of the previous plane of its own column (in
//     private shared-memory slots), so plane p-1 is updated as soon as the z-face p-1/2 is
//     solved in the pass over plane p.
// Primitives of planes p-1, p, p+1 (with a 2-cell ring) live in a 4-slot shared ring, into
// which three loader warps convert plane p+2 while plane p is computed; the raw conserved
// planes come in by TMA (interior columns) or cp.async (boundary columns). Every 9-field
// vector in shared memory is stored in float4 blocks (three instructions per vector). Each
// face is solved exactly once per CTA; the only recomputation is the Hancock state of the
// one-cell halo ring and the halo rows' y-faces.
// The new state's max signal speed (timestep.jl:4-14) is reduced in the same pass.
#pragma once
#include <cuda.h>  // CUtensorMap (the tiled-tensor descriptor the TMA loads read)

#include <type_traits>

#include "physics.cuh"

namespace pmf {

constexpr int TILE_X = 32;  // owned columns per CTA: one warp lane per column
constexpr int PLANE_W = 40; // staged plane width: x0-4 .. x0+35 (16-byte aligned rows for TMA)
constexpr int PLANE_X0 = 4; // column of x0 in the staged plane

// Threads per CTA: TY+2 row warps and the halo warp.
template <int TY> __host__ __device__ constexpr int step_warps() { return TY + 3; }
template <int TY> __host__ __device__ constexpr int step_threads() { return 32 * step_warps<TY>(); }
// The thread that issues the TMA loads and tracks the staging barrier's phase (a loader).
template <int TY> __host__ __device__ constexpr int step_stage_lead() { return 0; }
// CTAs per SM the step kernel is compiled for: short tiles fit two per SM (shared memory
// under half the SM's, registers capped at 128 per thread), so one CTA's barrier waits
// overlap the other's work.
template <int TY> __host__ __device__ constexpr int step_min_blocks() { return TY <= 5 ? 2 : 1; }
// Registers per thread the compiler may use: each of the SM's four sub-partitions holds 16K
// registers for the warps resident on it (ceil(warps / 4) per CTA times the CTAs per SM).
template <int TY> __host__ __device__ constexpr int step_reg_cap() {
  return 16384 / (32 * ((step_warps<TY>() + 3) / 4) * step_min_blocks<TY>()) / 8 * 8;
}

// Two staging buffers where shared memory allows (8 and 9 owned rows): the next plane's load is
// issued into the other buffer before the current one is converted, so the loaders need one
// barrier among themselves per plane instead of two. Shorter tiles must stay under half the
// SM's shared memory (two CTAs per SM), taller ones have no room.
template <int TY> __host__ __device__ constexpr bool step_double_stage() { return TY == 8 || TY == 9; }

// Number of CT workspace arrays written by the Godunov stage (reference CTState slots 4-15).
constexpr int CT_NWORK = 12;


struct StepArgs {
  const float* U[9];
  float* Un[9];
  float* resid[7];          // compensated mode: remainders of mx, my, mz, E, Bx, By, Bz
  const float* face[3];     // CT: lower-face normal B (bxf, byf, bzf)
  float* work[CT_NWORK];    // CT: mfx mfy mfz fxby fxbz fybx fybz fzbx fzby ecx ecy ecz
  int nx, ny, nz;
  int bc[3];
  int ntx, nty;             // column tiles along x and y
  float dtdx, ch, decay;
  Phys P;
  unsigned int* smax_bits;  // fused CFL reduction target (bits of a non-negative float), or null
  const float* dscal;       // if non-null: device {dtdx, ch, decay} overriding the values above
  unsigned int* status;     // device status bits (1: a bounded wait for a TMA load gave up), or null
  int use_tma;              // the tensor maps below describe U (fields with nx % 4 == 0)
  int tma_stall_polls;      // test hook, normally 0: > 0 arms each TMA plane's mbarrier without
                            // issuing its copies and gives up after this many polls, so the
                            // bounded-wait path runs with nothing in flight
  unsigned long long* census;  // RS_HLLD_CENSUS: solves, reference-degenerate and relative-only sides
  CUtensorMap tmap[9];      // per field: 3-D (x, y, z) FP32 map, box (PLANE_W, TY+4, 1)
  DragCoef drag;            // source-coupled steps: drag coefficients (read by SRC_DRAG/SRC_RAD kernels)
  int zlo, zhi;             // single-box launches: the planes [zlo, zhi) this launch updates
  float* corr;              // SRC_RAD: packed 9*nc correction buffer (slot 0 psi, 1-3 velocity
                            // corrections, 4 density increments, 5-7 B / 8 E remainders)
  int rad_flags;            // SRC_RAD: RAD_* bits
  const float* mask;        // SRC_RAD with RAD_MASKED: per-cell fallback mask (> 0: fall back)
};

// Source terms of the step (template parameter SRC of the step kernel).
enum { SRC_NONE = 0, SRC_DRAG = 1, SRC_RAD = 2 };
// Runtime options of the radiation-coupled step (StepArgs::rad_flags).
// RAD_FIRST_ORDER: zero reconstruction offsets in every cell, the piecewise-constant states of
// the cube kernel's global fallback (CHECK == 3, integrator_cube.jl:168-177).
// RAD_MASKED: the cube kernel's masked fallback (CHECK == 2, integrator_cube.jl:68-83,168-171):
// cells whose StepArgs::mask entry is positive take zero offsets, and every face with such a
// cell on either side is solved by LLF.
enum { RAD_TRACK_DENSITY = 1, RAD_TRACK_MAGNETIC = 2, RAD_TRACK_ENERGY = 4, RAD_CHECK = 8, RAD_FIRST_ORDER = 16,
       RAD_MASKED = 32 };

template <int TY>
struct StepSmem {
  static constexpr int PH = TY + 4;                 // rows y0-2 .. y0+TY+1
  static constexpr int PW = PLANE_W * PH;           // cells per staged plane
  static constexpr int PP = (PW + 31) / 32 * 32;    // staging field stride: 128-byte aligned for TMA
  static constexpr int STAGE = 9 * PP;              // raw conserved plane, [field][cell]
  static constexpr int NSTAGE = step_double_stage<TY>() ? 2 : 1;  // staging buffers
  // Primitive planes in blocks (fields 0-3 and 4-7 as one float4 per cell, field 8 as a float),
  // so a cell's nine values move in three shared-memory instructions. Rows are PRW = 42 cells
  // apart: the halo warp's lanes, which read two columns of eight rows, then hit distinct banks.
  static constexpr int PRW = 42;
  static constexpr int PPC = (PH * PRW + 3) / 4 * 4;  // cells per primitive plane (16-byte blocks)
  static constexpr int PRIM = 4 * 9 * PPC;          // 4-plane primitive ring
  static constexpr int G9 = 9 * 32;                 // one 9-vector per lane, in the same blocks
  static constexpr int YB = (TY + 1) * G9;          // y-face states / fluxes
  static constexpr int ZC = TY * 3 * G9;            // per owned thread: upper z state, lower z flux, x/y divergence
  static constexpr int YL = (TY + 1) * G9;          // lower y state of rows 1..TY+1, parked
  static constexpr int XB = TY * 9;                 // one x-face state or flux per owned row
  static constexpr int NL = 96;                     // loader threads: warps 0, TY+1 and the halo warp
  static constexpr int KL = (PW + NL - 1) / NL;     // staged entries per loader thread
  static constexpr int SI = 2 * KL * NL;            // per loader: source (x, y) offset; ring cell and flip bits
  static constexpr int FLOATS = NSTAGE * STAGE + PRIM + 2 * YB + ZC + YL + 3 * XB + SI;
  static constexpr size_t BYTES = sizeof(float) * FLOATS;
};

// Nine floats of one lane in a block group g of G9 floats: fields 0-3 at float4 [lane], fields
// 4-7 at float4 [32 + lane], field 8 at float [256 + lane]; every access is conflict-free.
__device__ __forceinline__ void st9g(float* g, int lane, const F9& v) {
  reinterpret_cast<float4*>(g)[lane] = make_float4(v[0], v[1], v[2], v[3]);
  reinterpret_cast<float4*>(g)[32 + lane] = make_float4(v[4], v[5], v[6], v[7]);
  g[256 + lane] = v[8];
}
__device__ __forceinline__ F9 ld9g(const float* g, int lane) {
  const float4 a = reinterpret_cast<const float4*>(g)[lane];
  const float4 b = reinterpret_cast<const float4*>(g)[32 + lane];
  return F9{{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, g[256 + lane]}};
}
// Nine fields of cell c of a primitive plane of NC cells (blocks of NC float4, NC float4, NC floats).
template <int NC> __device__ __forceinline__ void st9p(float* pl, int c, const F9& v) {
  reinterpret_cast<float4*>(pl)[c] = make_float4(v[0], v[1], v[2], v[3]);
  reinterpret_cast<float4*>(pl)[NC + c] = make_float4(v[4], v[5], v[6], v[7]);
  pl[8 * NC + c] = v[8];
}
template <int NC> __device__ __forceinline__ F9 ld9p(const float* pl, int c) {
  const float4 a = reinterpret_cast<const float4*>(pl)[c];
  const float4 b = reinterpret_cast<const float4*>(pl)[NC + c];
  return F9{{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, pl[8 * NC + c]}};
}

__device__ __forceinline__ void cp_async4(float* smem_dst, const float* gsrc) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// One column segment: planes [z0, z1) of column tile (tx, ty) of the box described by `a`.
// Every thread of the CTA calls it; `smax` accumulates the new state's max signal speed.
// TMA: the instantiation carries the bulk-tensor staging path (used where a.use_tma is set).
template <int TY, int RECON, int RSOL, bool CT, bool COMP, int SRC, bool TMA>
__device__ __forceinline__ void march_column(const StepArgs& a, int tx, int ty, int z0, int z1, float* smem,
                                             float& smax, unsigned long long* tma_bar, unsigned& tma_phase,
                                             int* tma_off, HlldCensus& cz) {
  constexpr bool DRAG = SRC != SRC_NONE;  // the radiation-coupled step always carries drag
  constexpr bool RAD = SRC == SRC_RAD;
  static_assert(!(DRAG && COMP), "source-coupled steps use their own remainders");
  using S = StepSmem<TY>;
  constexpr int NT = step_threads<TY>();
  constexpr int PP = S::PP;
  constexpr bool DSTAGE = step_double_stage<TY>();
  float* stage = smem;  // NSTAGE buffers of STAGE floats (each 128-byte aligned)
  float* prim = smem + S::NSTAGE * S::STAGE;
  // the staging buffer of plane zp (zp >= z0 - 2 >= -2)
  auto stage_of = [&](int zp) { return DSTAGE ? stage + ((zp + 4) & 1) * S::STAGE : stage; };
  // 9-vector groups (st9g / ld9g), 16-byte aligned: every size before them is a multiple of 4
  float* ybuf = prim + S::PRIM;    // [row] upper y state of rows 0..TY
  float* fybuf = ybuf + S::YB;     // [row-1] flux through the lower y face of rows 1..TY+1
  float* zcarry = fybuf + S::YB;   // [row][3] upper z state, lower z flux, x/y divergence of p-1
  float* ylow = zcarry + S::ZC;    // [row-1] lower y state of rows 1..TY+1
  float* xleft = ylow + S::YL;     // [row][9] upper x state of the left halo cell
  float* xright = xleft + S::XB;   // [row][9] upper x state of lane 31
  float* fxright = xright + S::XB; // [row][9] flux through the face above lane 31
  int* sidx = reinterpret_cast<int*>(fxright + S::XB);  // [KL][2][NL] staging map of this segment

  const int tid = threadIdx.x;
  const int lane = tid & 31, w = tid >> 5;
  const int x0 = tx * TILE_X, y0 = ty * TY;
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const int nxy = nx * ny;

  float dtdx = a.dtdx, ch = a.ch, decay = a.decay;
  if (a.dscal != nullptr) { dtdx = a.dscal[0]; ch = a.dscal[1]; decay = a.dscal[2]; }
  const float ich = 1.0f / ch;  // unused by CT (ch = 0)
  const Phys P = a.P;
  const float g = P.gamma;

  // row warps: cell (x0+lane, y0+w-1); halo warp lane t < 2*TY: row t/2, left (x0-1) or
  // right (x0+32) halo cell
  const bool halo_warp = w == TY + 2;
  const int hrow = lane >> 1, hside = lane & 1;
  const bool halo_act = halo_warp && lane < 2 * TY;
  const int x = halo_warp ? (hside ? x0 + TILE_X : x0 - 1) : x0 + lane;
  const int y = halo_warp ? y0 + hrow : y0 + w - 1;
  const bool row_own = w >= 1 && w <= TY;
  const bool own = row_own && x < nx && y < ny;

  // Staging is done by the three "loader" warps (the two y-halo rows and the halo warp),
  // which have the least solving to do: they prefetch plane p+3 and convert plane p+2 into
  // the primitive ring while the owned rows solve plane p.
  const bool loader = w == 0 || w >= TY + 1;
  const int lt = w == 0 ? lane : (w == TY + 1 ? 32 + lane : 64 + lane);
  // Staging map of this column: for each staged entry e (row r, column c) a loader handles,
  // the in-plane source offset iy*nx+ix under the x/y boundary rules, and the entry's cell in
  // the primitive ring (bits 2..) with the reflecting-wall flips (bit 0: x, bit 1: y). It is
  // the same for every plane, so it is built once per segment; per plane only the z index is
  // resolved.
  if (loader) {
#pragma unroll
    for (int k = 0; k < S::KL; ++k) {
      const int e = lt + k * S::NL;
      if (e < S::PW) {
        const int r = e / PLANE_W, c = e - r * PLANE_W;
        float fx, fy;
        const int ix = bc_index(x0 + c - PLANE_X0, nx, a.bc[0], &fx);
        const int iy = bc_index(y0 + r - 2, ny, a.bc[1], &fy);
        sidx[(2 * k) * S::NL + lt] = iy * nx + ix;
        sidx[(2 * k + 1) * S::NL + lt] = ((r * S::PRW + c) << 2) | (fx < 0.0f ? 1 : 0) | (fy < 0.0f ? 2 : 0);
      }
    }
  }
  // A plane whose staged box lies inside the grid comes in by TMA: one loader thread issues
  // nine tiled bulk-tensor loads (no multicast) that complete on an mbarrier. Other planes
  // (periodic wrap, outflow or reflecting ghosts) come in by per-element cp.async through the
  // staging map. After a bounded TMA wait has given up (*tma_off set), a late copy may still
  // land in `stage`, so the staging buffer is never touched again in this launch: every later
  // plane is converted straight from global memory.
  const bool tma_cols = TMA && a.use_tma && (__cvta_generic_to_shared(stage) & 127) == 0 && x0 - PLANE_X0 >= 0 &&
                        x0 - PLANE_X0 + PLANE_W <= nx && y0 - 2 >= 0 && y0 + TY + 2 <= ny;
  bool pending_tma = false;  // the plane in flight came by TMA
  const unsigned bar_addr = (unsigned)__cvta_generic_to_shared(tma_bar);
  auto issue_plane = [&](int zp) {  // loaders only
    pending_tma = false;
    if (*tma_off != 0) return;  // degraded staging: convert_plane reads global memory
    pending_tma = tma_cols && zp >= 0 && zp < nz;
    if (pending_tma) {
      if (lt == 0) {
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar_addr),
                     "r"((unsigned)(9 * S::PW * sizeof(float)))
                     : "memory");
#pragma unroll
        for (int f = 0; f < 9 && a.tma_stall_polls == 0; ++f) {
          const unsigned dst = (unsigned)__cvta_generic_to_shared(stage_of(zp) + f * PP);
          asm volatile(
              "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
              "[%5];\n" ::"r"(dst),
              "l"(reinterpret_cast<unsigned long long>(&a.tmap[f])), "r"(x0 - PLANE_X0), "r"(y0 - 2), "r"(zp),
              "r"(bar_addr)
              : "memory");
        }
      }
      return;
    }
    float fz;
    const int kz = bc_index(zp, nz, a.bc[2], &fz);
#pragma unroll
    for (int k = 0; k < S::KL; ++k) {
      const int e = lt + k * S::NL;
      if (e < S::PW) {
        const int gi = kz * nxy + sidx[(2 * k) * S::NL + lt];
#pragma unroll
        for (int f = 0; f < 9; ++f) cp_async4(stage_of(zp) + f * PP + e, a.U[f] + gi);
      }
    }
    cp_async_commit();
  };
  // Wait for the plane in flight (loaders only). A TMA wait is bounded: if the load never
  // lands, the status flag is raised and staging degrades to direct global loads for the rest
  // of the launch (the plane that timed out included), so the kernel always finishes and its
  // result is still the step's.
  const int poll_limit = a.tma_stall_polls > 0 ? a.tma_stall_polls : (1 << 22);
  auto wait_plane = [&]() {
    if (!pending_tma) {
      cp_async_wait_all();
      return;
    }
    unsigned done = 0;
    for (int it = 0; it < poll_limit && !done; ++it) {
      asm volatile(
          "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
          : "=r"(done)
          : "r"(bar_addr), "r"(tma_phase)
          : "memory");
    }
    if (!done) {
      *tma_off = 1;  // read by every loader after the next loader barrier
      if (lt == 0 && a.status != nullptr) atomicOr(a.status, 1u);
    }
    tma_phase ^= 1u;
  };
  // Raw conserved -> primitive (reflecting walls flip the normal components first); loaders.
  // The source is the staging buffer, or global memory once staging has degraded (one
  // uniform branch per plane; each source has its own loop).
  const bool reflect = a.bc[0] == BC_REFLECT || a.bc[1] == BC_REFLECT || a.bc[2] == BC_REFLECT;
  auto convert_from = [&](auto direct_tag, int zp, float* dst) {
    constexpr bool DIRECT = decltype(direct_tag)::value;
    const float* src = stage_of(zp);
    float fz;
    const int kz = bc_index(zp, nz, a.bc[2], &fz);
#pragma unroll
    for (int k = 0; k < S::KL; ++k) {
      const int e = lt + k * S::NL;
      if (e < S::PW) {
        const int fl = sidx[(2 * k + 1) * S::NL + lt];
        const float fx = (fl & 1) ? -1.0f : 1.0f, fy = (fl & 2) ? -1.0f : 1.0f;
        F9 u;
        if constexpr (DIRECT) {
          const int gi = kz * nxy + sidx[(2 * k) * S::NL + lt];
#pragma unroll
          for (int f = 0; f < 9; ++f) u[f] = __ldg(a.U[f] + gi);
        } else {
#pragma unroll
          for (int f = 0; f < 9; ++f) u[f] = src[f * PP + e];
        }
        if (reflect) {  // every flip is +1 without a reflecting wall
          u[1] *= fx; u[5] *= fx;
          u[2] *= fy; u[6] *= fy;
          u[3] *= fz; u[7] *= fz;
        }
        st9p<S::PPC>(dst, fl >> 2, cons2prim(u, g, P.smallr, P.pfl));
      }
    }
  };
  auto convert_plane = [&](int zp, float* dst) {
    if (*tma_off != 0) convert_from(std::true_type{}, zp, dst);
    else convert_from(std::false_type{}, zp, dst);
  };
  // barrier among the loader warps only (named barrier 1)
  auto loader_sync = [&]() { asm volatile("bar.sync 1, %0;\n" ::"r"(S::NL) : "memory"); };
  auto slot = [&](int zp) { return prim + ((zp - z0 + 4) & 3) * (9 * S::PPC); };
  auto ld9 = [&](const float* pl, int r, int c) { return ld9p<S::PPC>(pl, r * S::PRW + c); };

  // Prologue: primitives of planes z0-2, z0-1 and z0, plane z0+1 in flight.
  __syncthreads();  // the previous segment may still be reading shared memory
  if (loader) {
    if constexpr (DSTAGE) {
      issue_plane(z0 - 2);
      for (int zp = z0 - 2; zp <= z0; ++zp) {
        wait_plane();
        loader_sync();
        issue_plane(zp + 1);  // into the other buffer; zp + 1 <= z0 + 1 <= z1 + 1
        convert_plane(zp, slot(zp));
      }
    } else {
      for (int zp = z0 - 2; zp <= z0; ++zp) {
        issue_plane(zp);
        wait_plane();
        loader_sync();
        convert_plane(zp, slot(zp));
        loader_sync();
      }
      if (z0 + 1 <= z1 + 1) issue_plane(z0 + 1);
    }
  }

  // Per-column carries across planes (owned rows only), in this thread's private slots of
  // `zcarry`: the upper z-face state (ZC_STATE) and the lower z-face flux (ZC_FLUX) of plane p-1
  // and its x/y divergence ((Fxl - Fxh) + (Fyl - Fyh), ZC_DIV). Parking them in shared memory
  // keeps only the current solve's states in registers.
  enum { ZC_STATE = 0, ZC_FLUX = 1, ZC_DIV = 2 };
  float* zc = zcarry + (row_own ? (w - 1) : 0) * 3 * S::G9;
  auto zc_store = [&](int k, const F9& v) { st9g(zc + k * S::G9, lane, v); };
  auto zc_load = [&](int k) { return ld9g(zc + k * S::G9, lane); };
  // this thread's cell in the staged plane (halo lanes beyond 2*TY read a valid dummy cell)
  const int r0 = halo_warp ? (halo_act ? hrow + 2 : 2) : w + 1;
  const int c0 = halo_warp ? (hside ? PLANE_X0 + TILE_X : PLANE_X0 - 1) : PLANE_X0 + lane;

  // radiation: in-plane offset of this thread's cell, wrapped periodically (halo cells and
  // the columns/rows of a partial tile beyond the grid are periodic images)
  const int rad_xy = RAD ? (((y % ny) + ny) % ny) * nx + ((x % nx) + nx) % nx : 0;
  // masked fallback: the in-plane offsets of the cells on the lower x and y sides of this
  // cell's lower faces (periodic images), and the mask of this cell in the previous plane
  const bool masked = RAD && (a.rad_flags & RAD_MASKED) != 0;
  const int rad_xm = RAD ? (((y % ny) + ny) % ny) * nx + (((x - 1) % nx) + nx) % nx : 0;
  const int rad_ym = RAD ? ((((y - 1) % ny) + ny) % ny) * nx + ((x % nx) + nx) % nx : 0;

  // Where the register budget allows (TY = 8, 9: three warps per sub-partition), the state and
  // Kahan remainders of the next plane this thread updates are loaded one pass ahead, so their
  // HBM/L2 latency overlaps a whole pass of flux work instead of stalling the update; under a
  // 128-register cap the 16 extra live values would spill, and the update loads them itself.
  constexpr bool PREFETCH = step_reg_cap<TY>() >= 160;
  constexpr int NR = COMP ? (CT ? 4 : 7) : 1;
  F9 u0;
  float rk[NR];
  auto prefetch_cell = [&](int pz) {
    const int c = pz * nxy + y * nx + x;
#pragma unroll
    for (int f = 0; f < 9; ++f) u0[f] = __ldg(a.U[f] + c);
    if constexpr (COMP) {
#pragma unroll
      for (int i = 0; i < NR; ++i) rk[i] = a.resid[i][c];
    }
  };
  // Conservative update of cell (x, y, pz) from its x/y divergence and its two z fluxes
  // (u0 and rk hold that cell: loaded by prefetch_cell(pz) during the previous pass, or here).
  auto update_cell = [&](int pz, const F9& dxy, const F9& flo, const F9& fhi) {
    const int c = pz * nxy + y * nx + x;
    if constexpr (!PREFETCH) prefetch_cell(pz);
    F9 un;
    float d[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) d[i] = dtdx * (dxy[i] + (flo[i] - fhi[i]));
    un[0] = u0[0] + d[0];
    if constexpr (COMP) {
#pragma unroll
      for (int i = 1; i <= NR; ++i) {
        float r = rk[i - 1];
        un[i] = comp_add(u0[i], d[i], r);
        a.resid[i - 1][c] = r;
      }
      if constexpr (CT) {
#pragma unroll
        for (int i = NR + 1; i <= 7; ++i) un[i] = u0[i] + d[i];
      }
    } else {
#pragma unroll
      for (int i = 1; i <= 7; ++i) un[i] = u0[i] + d[i];
    }
    if constexpr (RAD) {
      // radiation-coupled update (integrator_cube.jl:85-106,412-436; integrator_ref.jl:140-156):
      // density increment accumulated, E and (GLM) cell B through their Kahan remainders,
      // admissibility flag, drag corrector with E's remainder; negative density marks a
      // rejected cell
      const size_t n = (size_t)nxy * nz, cc = (size_t)c;
      const int fl = a.rad_flags;
      float* cr = a.corr;
      if (fl & RAD_TRACK_DENSITY) cr[4 * n + cc] += d[0];
      float rE = (fl & RAD_TRACK_ENERGY) ? cr[8 * n + cc] : 0.0f;
      if (fl & RAD_TRACK_ENERGY) un[4] = comp_add(u0[4], d[4], rE);
      if (!CT && (fl & RAD_TRACK_MAGNETIC)) {
#pragma unroll
        for (int i = 5; i <= 7; ++i) {
          float r = cr[(size_t)i * n + cc];
          un[i] = comp_add(u0[i], d[i], r);
          cr[(size_t)i * n + cc] = r;
        }
      }
      un[8] = u0[8] + d[8];
      const bool bad = (fl & RAD_CHECK) && inadmissible_cell(un, P);
      drag_correct_cell(u0, un, a.drag, P.smallr, (fl & RAD_TRACK_ENERGY) ? &rE : nullptr);
      if (fl & RAD_TRACK_ENERGY) cr[8 * n + cc] = rE;
      if (bad) un[0] = -fmaxf(fabsf(un[0]), fmaxf(P.smallr, P.llf_dmin));
    } else if constexpr (DRAG) {
      // drag corrector on the uncompensated trial (its energy floor reads the trial cell B,
      // which CT later replaces by the face average); integrator_ref.jl:155-156
      drag_correct_cell(u0, un, a.drag, P.smallr);
    }
    un[8] = CT ? 0.0f : (u0[8] + d[8]) * decay;
#pragma unroll
    for (int f = 0; f < 9; ++f) {
      if (CT && f >= 5 && f <= 7) continue;  // cell B comes from the face average
      a.Un[f][c] = un[f];
    }
    if (!CT && a.smax_bits != nullptr) smax = fmaxf(smax, cell_wavespeed(un, P));
  };
  // Staggered normal field of this thread's cell's lower face along axis D (CT, periodic).
  // x, y and pz are at most one period outside the box, so one conditional wrap suffices.
  auto wrap1 = [](int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); };
  auto face_bn = [&](int D, int pz) {
    return __ldg(a.face[D] + wrap1(pz, nz) * nxy + wrap1(y, ny) * nx + wrap1(x, nx));
  };
  // fallback mask of in-plane offset xy in plane pz (periodic: pz is at most one period out)
  auto mask_at = [&](int pz, int xy) { return __ldg(a.mask + (size_t)wrap1(pz, nz) * nxy + xy) > 0.0f; };
  bool m_zlo = false;  // mask of this cell in plane p-1 (the lower side of its z-face)

  F9 Fx;  // this thread's lower x-face flux of the last owned plane solved
  for (int p = z0 - 1; p <= z1; ++p) {
    __syncthreads();  // plane p+1 (converted during the previous pass) is in the ring; the x/y
                      // fluxes of plane p-1 are complete
    // x/y flux divergence of plane p-1 for the owned rows, parked for its update in the z-solve
    // of this pass (the face above lane 31 comes from the halo warp)
    if (row_own && p > z0) {
      F9 dxy;
      const F9 fyl = ld9g(fybuf + (w - 1) * S::G9, lane), fyh = ld9g(fybuf + w * S::G9, lane);
#pragma unroll
      for (int i = 0; i < 9; ++i) {
        const float dn = __shfl_down_sync(0xffffffffu, Fx[i], 1);
        const float fxh = lane == TILE_X - 1 ? fxright[(w - 1) * 9 + i] : dn;
        dxy[i] = (Fx[i] - fxh) + (fyl[i] - fyh[i]);
      }
      zc_store(ZC_DIV, dxy);
    }
    const bool mid = p >= z0 && p < z1;  // an owned plane of this chunk
    const int cell_p = (mid && x < nx && y < ny) ? (p * nxy + y * nx + x) : 0;
    // this thread's Hancock state and face offsets of plane p, and (CT) its lower-face fields
    F9 mh;
    Offsets<RECON> ox, oy, oz;
    float bnx = 0.0f, bny = 0.0f, bnz = 0.0f;
    bool m_c = false;  // masked fallback: this cell of plane p is masked
    // planes z0-1 and z1 only feed the chunk's end z-faces: only the owned rows work on them
    if (mid || row_own) {

    // CT: the staggered normal fields of this cell's three lower faces, fetched now so that
    // their latency overlaps the Hancock step (x: all solving lanes; y: rows 1..TY+1; z:
    // owned rows)
    if constexpr (CT) {
      if (p >= z0 && p < z1) {
        if (row_own || (halo_act && hside == 1)) bnx = face_bn(0, p);
        if (w >= 1 && !halo_warp) bny = face_bn(1, p);
      }
      if (row_own) bnz = face_bn(2, p);
    }

    // ---- Hancock half step of this thread's cell in plane p ------------------------------
    const float* pm = slot(p - 1);
    const float* p0 = slot(p);
    const float* pp = slot(p + 1);
    const F9 m0 = ld9(p0, r0, c0);
    ox = recon<RECON>(ld9(p0, r0, c0 - 1), m0, ld9(p0, r0, c0 + 1));
    oy = recon<RECON>(ld9(p0, r0 - 1, c0), m0, ld9(p0, r0 + 1, c0));
    oz = recon<RECON>(ld9(pm, r0, c0), m0, ld9(pp, r0, c0));
    if constexpr (RAD) {
      // piecewise-constant states: every offset replaced by zero (m0 + 0 == m0, so every face
      // state and Hancock flux difference is that of zero offsets), without a branch
      // (all cells under the global fallback, masked cells under the masked one)
      m_c = masked && mask_at(p, rad_xy);
      const bool keep = (a.rad_flags & RAD_FIRST_ORDER) == 0 && !m_c;
      keep_offsets(ox, keep);
      keep_offsets(oy, keep);
      keep_offsets(oz, keep);
    }
    {
      const F9 u0 = prim2cons(m0, g);
      F9 acc = hancock_term<0, RECON>(m0, ox, g);
      acc = add9(acc, hancock_term<1, RECON>(m0, oy, g));
      acc = add9(acc, hancock_term<2, RECON>(m0, oz, g));
      const float h = 0.5f * dtdx;
      F9 uh;
#pragma unroll
      for (int i = 0; i < 9; ++i) uh[i] = u0[i] - h * acc[i];
      mh = cons2prim(uh, g, P.smallr, P.pfl);
    }
    // drag: face states and the CT cell EMF see the drag-propagated velocity
    // (integrator_ref.jl:28-31,135)
    if constexpr (DRAG) drag_predict_cell<RECON>(mh, m0, ox, oy, oz, a.drag);
    // radiation: the cell's velocity correction is added to all its face states and to the
    // CT cell EMF velocity (integrator_ref.jl:33-39,135); its periodic image for halo cells
    if constexpr (RAD) {
      if (!halo_warp || halo_act) {
        const size_t n = (size_t)nxy * nz;
        const size_t gi = (size_t)wrap1(p, nz) * nxy + rad_xy;
        mh[1] += __ldg(a.corr + n + gi);
        mh[2] += __ldg(a.corr + 2 * n + gi);
        mh[3] += __ldg(a.corr + 3 * n + gi);
      }
    }
    if constexpr (CT) {
      // cell-centred reference EMF -v x B: v of the predicted state, B at the start of the
      // step (integrator_ref.jl:133-138)
      if (own && mid) {
        a.work[9][cell_p] = mh[3] * m0[6] - mh[2] * m0[7];
        a.work[10][cell_p] = mh[1] * m0[7] - mh[3] * m0[5];
        a.work[11][cell_p] = mh[2] * m0[5] - mh[1] * m0[6];
      }
    }
    if (p == z0 - 1) {
      zc_store(ZC_STATE, face_hi<RECON>(mh, oz));
      m_zlo = m_c;
    } else {
    if (mid && !halo_warp) {
      // upper y state for the row above (row warps 0..TY); lower y state parked (rows 1..TY+1)
      if (w <= TY) st9g(ybuf + w * S::G9, lane, face_hi<RECON>(mh, oy));
      if (w >= 1) st9g(ylow + (w - 1) * S::G9, lane, face_lo<RECON>(mh, oy));
    }
    // x-face states at the tile edges go through shared memory
    if (mid && row_own && lane == TILE_X - 1) {
      const F9 xR = face_hi<RECON>(mh, ox);
#pragma unroll
      for (int i = 0; i < 9; ++i) xright[(w - 1) * 9 + i] = xR[i];
    }
    if (mid && halo_act && hside == 0) {
      const F9 xR = face_hi<RECON>(mh, ox);
#pragma unroll
      for (int i = 0; i < 9; ++i) xleft[hrow * 9 + i] = xR[i];
    }
    if (row_own) {
      // ---- z-face p-1/2: left = carried upper z state of p-1, right = lower z state of p --
      F9 L = zc_load(ZC_STATE), R = face_lo<RECON>(mh, oz);
      zc_store(ZC_STATE, face_hi<RECON>(mh, oz));
      if constexpr (CT) {
        L[7] = bnz; R[7] = bnz;
      }
      const F9 Fz = riemann<2, RSOL, CT>(L, R, ch, ich, P, (own && mid) ? &cz : nullptr, m_zlo || m_c);
      m_zlo = m_c;
      if constexpr (CT) {
        if (own && mid) {
          a.work[2][cell_p] = Fz[0];
          a.work[7][cell_p] = Fz[5];
          a.work[8][cell_p] = Fz[6];
        }
      }
      if (p > z0 && own) update_cell(p - 1, zc_load(ZC_DIV), zc_load(ZC_FLUX), Fz);
      if constexpr (PREFETCH) {
        if (mid && own) prefetch_cell(p);
      }
      zc_store(ZC_FLUX, Fz);
    }
    }  // p > z0 - 1
    }  // mid || row_own
    // ---- loaders: convert plane p+2 (its ring slot last held p-2) and prefetch p+3 -----------
    if (loader && p + 2 <= z1 + 1) {
      wait_plane();
      loader_sync();
      if constexpr (DSTAGE) {
        // the other buffer was last read by convert(p+1), which every loader finished before
        // this barrier
        if (p + 3 <= z1 + 1) issue_plane(p + 3);
        convert_plane(p + 2, slot(p + 2));
      } else {
        convert_plane(p + 2, slot(p + 2));
        loader_sync();
        if (p + 3 <= z1 + 1) issue_plane(p + 3);
      }
    }
    if (!mid) continue;  // p == z0-1 or z1: only the chunk's end z-faces and update were needed
    __syncthreads();

    // ---- x-faces: lane l of a row warp solves the face below column l (lane 0 against the
    // left halo cell); the halo warp's right-side lanes solve the face above lane 31. Both
    // go through this one call site, so a face shared by two tiles gets the same bits.
    {
      F9 L, R = face_lo<RECON>(mh, ox);
      {
        const F9 xR = face_hi<RECON>(mh, ox);
#pragma unroll
        for (int i = 0; i < 9; ++i) L[i] = __shfl_up_sync(0xffffffffu, xR[i], 1);
      }
      if (row_own || (halo_act && hside == 1)) {
#pragma unroll
        for (int i = 0; i < 9; ++i)
          if (halo_warp) L[i] = xright[hrow * 9 + i];
          else if (lane == 0) L[i] = xleft[(w - 1) * 9 + i];
        if constexpr (CT) {
          L[5] = bnx; R[5] = bnx;
        }
        Fx = riemann<0, RSOL, CT>(L, R, ch, ich, P, own ? &cz : nullptr, masked && (m_c || mask_at(p, rad_xm)));
        if (halo_warp) {
#pragma unroll
          for (int i = 0; i < 9; ++i) fxright[hrow * 9 + i] = Fx[i];
        }
        if constexpr (CT) {
          if (own) {
            a.work[0][cell_p] = Fx[0];
            a.work[3][cell_p] = Fx[6];
            a.work[4][cell_p] = Fx[7];
          }
        }
      }
    }
    // ---- y-faces: rows 1..TY+1 solve the face below them from two shared-memory states ---
    if (w >= 1 && !halo_warp) {
      F9 L = ld9g(ybuf + (w - 1) * S::G9, lane), R = ld9g(ylow + (w - 1) * S::G9, lane);
      if constexpr (CT) {
        L[6] = bny; R[6] = bny;
      }
      const F9 Fy = riemann<1, RSOL, CT>(L, R, ch, ich, P, own ? &cz : nullptr, masked && (m_c || mask_at(p, rad_ym)));
      st9g(fybuf + (w - 1) * S::G9, lane, Fy);
      if constexpr (CT) {
        if (own) {
          a.work[1][cell_p] = Fy[0];
          a.work[5][cell_p] = Fy[5];
          a.work[6][cell_p] = Fy[7];
        }
      }
    }
  }
  cp_async_wait_all();
}

// After the last plane: if a bounded TMA wait gave up in this launch, give the copies of that
// plane one more bounded wait before the CTA exits (its shared memory may not be released with
// a bulk copy still writing into it). Every thread of the CTA calls it; thread `lead`, a
// loader, tracks the barrier phase.
__device__ __forceinline__ void drain_tma(unsigned long long* bar, unsigned tma_phase, const int* off, int polls,
                                          int lead) {
  __syncthreads();
  if ((int)threadIdx.x != lead || *off == 0) return;
  const unsigned addr = (unsigned)__cvta_generic_to_shared(bar);
  unsigned done = 0;
  for (int it = 0; it < polls && !done; ++it) {
    asm volatile(
        "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(addr), "r"(tma_phase ^ 1u)
        : "memory");
  }
}

// Census counts of the CTA summed into census[0..2] (every thread calls it).
__device__ __forceinline__ void flush_census(const HlldCensus& cz, unsigned long long* census) {
  unsigned long long v[3] = {cz.solves, cz.ref_sides, cz.rel_sides};
#pragma unroll
  for (int q = 0; q < 3; ++q) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
    if ((threadIdx.x & 31) == 0 && v[q] != 0) atomicAdd(census + q, v[q]);
  }
}

// The staging mbarrier (one arrival per TMA plane, the loads' bytes as its transaction).
__device__ __forceinline__ void init_tma_barrier(unsigned long long* bar, int* off) {
  if (threadIdx.x == 0) {
    *off = 0;
    const unsigned addr = (unsigned)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(addr) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
}

// Block-wide max of v and one atomicMax into *bits (every thread of the CTA calls it).
template <int NT>
__device__ __forceinline__ void flush_smax(float v, unsigned int* bits) {
  __shared__ float red[32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  v = warp_max(v);
  if (lane == 0) red[w] = v;
  __syncthreads();
  if (w == 0) {
    v = lane < NT / 32 ? red[lane] : 0.0f;
    v = warp_max(v);
    if (lane == 0) atomicMax(bits, __float_as_uint(v));
  }
}

// Planes [q0, q1) of a (column, plane) index space, q = column * nz + z, split into column
// segments: CTA b of B takes [b*Q/B, (b+1)*Q/B), so every CTA does the same number of
// planes (to within one) and the launch has no partial last wave.
__device__ __forceinline__ void cta_range(long long Q, long long* q0, long long* q1) {
  *q0 = Q * blockIdx.x / gridDim.x;
  *q1 = Q * (blockIdx.x + 1) / gridDim.x;
}

// One box: a persistent launch of one CTA per resident slot. The plain and compensated GLM
// instantiations stage interior planes by TMA; the CT and source-coupled ones are compiled
// without the TMA path and stage every plane by cp.async: the path's code cost them 4 % (CT,
// 2.38 against 2.29 ms per 256^3 step), 2 % (drag) and 5 % (radiation), the GLM step 0.5 %.
template <int TY, int RECON, int RSOL, bool CT, bool COMP, int SRC>
__global__ void __launch_bounds__(step_threads<TY>(), step_min_blocks<TY>()) mhd_step_kernel(const __grid_constant__ StepArgs a) {
  extern __shared__ __align__(128) float smem[];
  __shared__ unsigned long long tma_bar;
  __shared__ int tma_off;
  unsigned tma_phase = 0;
  init_tma_barrier(&tma_bar, &tma_off);
  long long q, qe;
  const int nzr = a.zhi - a.zlo;  // planes of this launch
  cta_range((long long)a.ntx * a.nty * nzr, &q, &qe);
  float smax = 0.0f;
  HlldCensus cz{0u, 0u, 0u};
  while (q < qe) {
    const int col = (int)(q / nzr);
    const int zr = (int)(q - (long long)col * nzr);
    const int z0 = a.zlo + zr;
    const int z1 = a.zlo + (int)min((long long)nzr, zr + (qe - q));
    march_column<TY, RECON, RSOL, CT, COMP, SRC, !CT && SRC == SRC_NONE>(a, col % a.ntx, col / a.ntx, z0, z1, smem, smax, &tma_bar,
                                                  tma_phase, &tma_off, cz);
    q += z1 - z0;
  }
  drain_tma(&tma_bar, tma_phase, &tma_off, a.tma_stall_polls > 0 ? a.tma_stall_polls : (1 << 22),
            step_stage_lead<TY>());
  if constexpr (RSOL == RS_HLLD_CENSUS) flush_census(cz, a.census);
  if (!CT && a.smax_bits != nullptr) flush_smax<step_threads<TY>()>(smax, a.smax_bits);
}

// Many boxes in one launch: box b owns global indices [q0_b, q0_{b+1}) of the concatenated
// (column, plane) spaces; each CTA walks its equal share across box boundaries. Compiled
// without the TMA path, every plane staged by cp.async: with it the batch kernel sat at its
// register cap (168 against 158) and one 256^3 box took 2.06 ms per step against 1.82 ms.
struct alignas(64) BoxStep {
  StepArgs a;     // per-box pointers, extents and parameters; dscal = that box's {dt/dx, ch, decay}
  long long q0;   // first global (column, plane) index of this box
};

template <int TY, int RECON, int RSOL, bool CT, bool COMP>
__global__ void __launch_bounds__(step_threads<TY>(), step_min_blocks<TY>()) mhd_batch_kernel(const BoxStep* __restrict__ boxes, int nbox,
                                                                       long long Q) {
  extern __shared__ __align__(128) float smem[];
  __shared__ unsigned long long tma_bar;
  __shared__ int tma_off;
  unsigned tma_phase = 0;
  long long q, qe;
  cta_range(Q, &q, &qe);
  if (q >= qe) return;
  init_tma_barrier(&tma_bar, &tma_off);
  int b = 0, hi = nbox - 1;
  while (b < hi) {  // last box with q0 <= q
    const int mid = (b + hi + 1) >> 1;
    if (boxes[mid].q0 <= q) b = mid;
    else hi = mid - 1;
  }
  float smax = 0.0f;
  HlldCensus cz{0u, 0u, 0u};  // unused: the batched form has no census
  while (q < qe) {
    while (b + 1 < nbox && boxes[b + 1].q0 <= q) {
      if (!CT && boxes[b].a.smax_bits != nullptr) flush_smax<step_threads<TY>()>(smax, boxes[b].a.smax_bits);
      smax = 0.0f;
      ++b;
    }
    const StepArgs& a = boxes[b].a;
    const long long local = q - boxes[b].q0;
    const int col = (int)(local / a.nz);
    const int z0 = (int)(local - (long long)col * a.nz);
    const int z1 = (int)min((long long)a.nz, z0 + (qe - q));
    march_column<TY, RECON, RSOL, CT, COMP, SRC_NONE, false>(a, col % a.ntx, col / a.ntx, z0, z1, smem, smax, &tma_bar,
                                                   tma_phase, &tma_off, cz);
    q += z1 - z0;
  }
  drain_tma(&tma_bar, tma_phase, &tma_off, 1 << 22, step_stage_lead<TY>());
  if (!CT && boxes[b].a.smax_bits != nullptr) flush_smax<step_threads<TY>()>(smax, boxes[b].a.smax_bits);
}

}  // namespace pmf
