/*
 * pmfmhd.h — C ABI of libpmfmhd.so, a B200 (sm_100a) implementation of the PMFGLM
 * ideal-MHD Godunov step (MUSCL-Hancock, MC-PLM / PPM / minmod reconstruction,
 * HLLD / HLL / LLF Riemann solvers, Dedner GLM cleaning or face-staggered CT).
 *
 * Every field pointer is a DEVICE pointer to caller-owned FP32 storage in the
 * reference's SoA layout: nine arrays U = (rho, rho*vx, rho*vy, rho*vz, E, Bx, By, Bz, psi)
 * of nc = nx*ny*nz values each, cell (i,j,k) (0-based) at ((k*ny)+j)*nx+i (x fastest),
 * exactly MHDKernels' `linidx` (lib/MHDKernels/src/state.jl:95). The library never frees
 * caller memory; it allocates only small internal workspace owned by a pmfmhd_ctx.
 *
 * All calls return 0 on success or a negative PMFMHD_E* code (pmfmhd_strerror). Work is
 * enqueued on the caller's stream (a cudaStream_t passed as void*; NULL = legacy default
 * stream). Calls whose result is a host value synchronise that stream before returning.
 */
#ifndef PMFMHD_H
#define PMFMHD_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PMFMHD_OK 0
#define PMFMHD_EINVAL (-1)        /* null pointer, unknown code, non-finite scalar */
#define PMFMHD_ESHAPE (-2)        /* grid extent out of range */
#define PMFMHD_ECUDA (-3)         /* CUDA runtime error (message: pmfmhd_last_cuda_error) */
#define PMFMHD_ETIMEOUT (-4)      /* a bounded device-side wait gave up */
#define PMFMHD_EINADMISSIBLE (-5) /* non-finite / non-positive state found by a check */
#define PMFMHD_ENOMEM (-6)        /* workspace allocation failed */
#define PMFMHD_EUNSUPPORTED (-7)  /* combination not provided (e.g. CT with non-periodic BCs) */

/* Reconstruction codes (glm_physics.jl:202-207). */
#define PMFMHD_RECON_PLM 0        /* MonCen (MC) PLM */
#define PMFMHD_RECON_PPM 1        /* local CW84 PPM */
#define PMFMHD_RECON_PLM_MINMOD 2 /* minmod PLM */
/* Riemann solver codes (glm_physics.jl:309-314). */
#define PMFMHD_RIEMANN_HLLD 0
#define PMFMHD_RIEMANN_HLL 1
#define PMFMHD_RIEMANN_LLF 2
/* Boundary codes (boundary.jl:152-159). */
#define PMFMHD_BC_PERIODIC 0
#define PMFMHD_BC_OUTFLOW 1
#define PMFMHD_BC_REFLECT 2

/* HLLD single-star degeneracy tolerances (pmfmhd_grid.hlld_dtol_rel). */
#define PMFMHD_HLLD_DTOL_REFERENCE 0.0f /* the reference's test |denK| < 1e-12 */
#define PMFMHD_HLLD_DTOL_RELATIVE 1e-5f /* |denK| < max(1e-12, 1e-5 bn^2) */

/* Grid and run parameters: the scalar fields of MHDState (state.jl:63-79), plus the HLLD
 * degeneracy tolerance. */
typedef struct pmfmhd_grid {
  int32_t nx, ny, nz;
  int32_t bc[3];   /* per axis, PMFMHD_BC_* */
  int32_t recon;   /* PMFMHD_RECON_* */
  int32_t riemann; /* PMFMHD_RIEMANN_* */
  float dx, gamma, smallr, pfl, llf_dmin, llf_pmin;
  /* HLLD single-star states (glm_physics.jl:255-263) fall back to the unmodified transverse
   * state when |denK| < max(1e-12, hlld_dtol_rel * bn^2), denK = d(S-u)(S-SM) - bn^2.
   * 0 (PMFMHD_HLLD_DTOL_REFERENCE) is the reference's own absolute test |denK| < 1e-12: the
   * reference's arithmetic exactly. 1e-5 (PMFMHD_HLLD_DTOL_RELATIVE) widens it to the FP32
   * rounding level of denK, where the single-star states are otherwise ~1/denK of rounding
   * noise; it changes the flux only at those near-degenerate faces (a handful per step on a
   * turbulent 256^3 box) and kept a 512^3 turbulent box finite that blew up with the absolute
   * test. Must be finite and >= 0. */
  float hlld_dtol_rel;
} pmfmhd_grid;

/* Opaque per-device context: reduction workspace, tile autotuning table, cached graphs. */
typedef struct pmfmhd_ctx pmfmhd_ctx;

/* Library version (major*10000 + minor*100 + patch). */
int pmfmhd_version(void);
const char* pmfmhd_strerror(int code);
/* Text of the last CUDA error seen by this thread (empty if none). */
const char* pmfmhd_last_cuda_error(void);

/* Create / destroy a context on CUDA device `device` (the device is made current). */
int pmfmhd_create(int device, pmfmhd_ctx** out);
int pmfmhd_destroy(pmfmhd_ctx* ctx);

/*
 * One GLM Godunov step: read U, write Unew (distinct buffers), psi damped by `decay`.
 * Replaces the KernelAbstractions launch `_cube_launch!(Val(:raw), CUDABackend, s, dt, ch, decay)`
 * (lib/MHDKernels/ext/MHDKernelsCUDAExt.jl:22-26, integrator_cube.jl:467-476) and equally
 * `step_ref!` (integrator_ref.jl:210-220): U = s.U, Unew = s.scratch; the caller swaps.
 * dt is the step, ch the GLM cleaning speed, decay = exp(-cr*ch*dt/dx) (driver.jl:29).
 * resid: NULL for the plain FP32 update, or 7 device arrays of Kahan remainders
 * (rho*vx, rho*vy, rho*vz, E, Bx, By, Bz), zero-initialised by the caller and kept across
 * steps (compensated update, glm_physics.jl:349-359, extended to momentum).
 * The new state's max signal speed max(|v_d| + c_f,d) is reduced in the same launch and
 * can be read with pmfmhd_last_wavespeed.
 */
int pmfmhd_step_glm(pmfmhd_ctx* ctx, const pmfmhd_grid* g, const float* const U[9], float* const Unew[9],
                    float dt, float ch, float decay, float* const resid[7], void* stream);

/*
 * The GLM step of pmfmhd_step_glm on HOST buffers: Uh (9 host arrays) in, Unh (9 host arrays)
 * out, for a caller whose state lives in host memory (the reference's CPU-resident
 * `MHDState`, whose `step_ref!` this replaces for that case). The box is cut into `nchunks`
 * z-slabs (<= 0: 16; each at least 2 planes): slabs are copied in on one stream, stepped on a
 * second once their neighbours have arrived, and copied out on a third, so the PCIe traffic
 * both ways overlaps the compute. Pinned host memory (cudaHostAlloc / cudaHostRegister) is
 * needed for the overlap; pageable memory works, serialised. Nine arrays spaced one field
 * apart (a (9, cells) block) move as one pitched copy per slab. Ordered after the caller's
 * stream; returns after Unh is complete. Device copies of the state are context workspace
 * (18 floats per cell, kept for the next call). No compensation (resid is not supported).
 */
int pmfmhd_step_glm_host(pmfmhd_ctx* ctx, const pmfmhd_grid* g, const float* const Uh[9], float* const Unh[9],
                         float dt, float ch, float decay, int nchunks, void* stream);

/*
 * One constrained-transport step (mhd_solver=:ct): Godunov stage with the staggered
 * normal field on every face, Gardiner-Stone 2005 edge EMFs, face curl update and the
 * face-averaged cell B. Replaces `step!`'s CT branch: `step_ref!(s, dt; ch=0, decay=1)`
 * followed by `ct_update!` (driver.jl:22-27, integrator_ref.jl:210-220, ct.jl:158-173).
 * ct_packed is the reference's CTState buffer (state.jl:44-58): 21*nc floats, slots
 * bxf,byf,bzf | mfx,mfy,mfz | fxby,fxbz,fybx,fybz,fzbx,fzby | ecx,ecy,ecz | ex,ey,ez |
 * rbx,rby,rbz. Slots 0-2 are updated in place, 3-17 are workspace, 18-20 hold the face
 * Kahan remainders used when compensate_faces != 0. Requires all-periodic boundaries.
 * resid: NULL or 7 remainder arrays as for pmfmhd_step_glm (the B slots are unused).
 */
int pmfmhd_step_ct(pmfmhd_ctx* ctx, const pmfmhd_grid* g, const float* const U[9], float* const Unew[9],
                   float* ct_packed, float dt, float* const resid[7], int compensate_faces, void* stream);

/*
 * Source-coupled drag step: the GLM Godunov step above with linear (Compton) drag of
 * impulse q = drag_impulse = Gamma*dt toward target_velocity (null = at rest) folded in.
 * Replaces `step_ref_drag!` (integrator_ref.jl:222-234) and `step_cube_drag!`
 * (integrator_cube.jl:478-490), the kernels behind `step_drag_godunov!` (drag.jl:162-178):
 * the Hancock face states (and the CT cell EMF) carry the drag-propagated velocity
 * v0 + exp(-q/2)(v - v0) + phi1(q/2)(v_half - v) (glm_physics.jl:71-84), and each cell's
 * trial update is corrected by the exact momentum response and the integrated drag work
 * (`drag_correct_conserved`, glm_physics.jl:128-172). No compensation (the reference passes
 * no tracking flags), so a compensated state's remainders are left untouched.
 * q must be finite and >= 0 (PMFMHD_EINVAL otherwise); q = 0 gives the plain step up to
 * the density floor max(rho, smallr) of the corrector.
 */
int pmfmhd_step_glm_drag(pmfmhd_ctx* ctx, const pmfmhd_grid* g, const float* const U[9], float* const Unew[9],
                         float dt, float ch, float decay, float drag_impulse, const float target_velocity[3],
                         void* stream);
/* The CT form (step_ref_drag! on a mhd_solver=:ct state, then ct_update! without face
 * compensation, integrator_ref.jl:222-234). */
int pmfmhd_step_ct_drag(pmfmhd_ctx* ctx, const pmfmhd_grid* g, const float* const U[9], float* const Unew[9],
                        float* ct_packed, float dt, float drag_impulse, const float target_velocity[3],
                        void* stream);
/* Options of pmfmhd_step_radiation (bitwise or). */
#define PMFMHD_RAD_TRACK_DENSITY 1         /* accumulate the density increments in slot 4 */
#define PMFMHD_RAD_TRACK_MAGNETIC 2        /* Kahan-compensate cell B (GLM, slots 5-7) or the CT faces */
#define PMFMHD_RAD_TRACK_ENERGY 4          /* Kahan-compensate E and the drag work (slot 8) */
#define PMFMHD_RAD_CHECK_ADMISSIBILITY 8   /* write -max(|rho|, max(smallr, llf_dmin)) for rejected cells */
#define PMFMHD_RAD_ROBUST_FALLBACK 16      /* minmod PLM with HLL on every face */
#define PMFMHD_RAD_GLOBAL_FALLBACK 32      /* piecewise-constant states and LLF on every face, with the admissibility check */
#define PMFMHD_RAD_MASKED_FALLBACK 64      /* per-cell mask in slot 4: masked cells piecewise constant, their faces LLF */
/*
 * Radiation-coupled step: the drag step (target at rest, impulse drag_impulse) whose face
 * states also carry a per-cell velocity correction, with optional tracking of the density
 * increment and Kahan remainders of E and B. Replaces `step_ref_radiation!`
 * (integrator_ref.jl:238-258; GLM and CT) and `step_cube_radiation!`
 * (integrator_cube.jl:504-540; check_admissibility, global_fallback and robust_fallback).
 * `correction` is the caller's packed buffer of 9*nc floats, as the reference's
 * `packed_psi_correction`: slot 0 holds psi and is read in place of U[8] (which may be
 * null), slots 1-3 the velocity corrections added to every face state of their cell (and to
 * the CT cell EMF velocity), slot 4 receives the density increments, slots 5-7 and 8 are
 * the remainders of cell B (GLM) and E. For CT states (ct_packed non-null) ch and decay are
 * ignored and the faces are compensated when PMFMHD_RAD_TRACK_MAGNETIC is set. Requires
 * all-periodic boundaries.
 * PMFMHD_RAD_MASKED_FALLBACK is the cube kernel's masked fallback (`fallback=true`, launched
 * with CHECK == 2, integrator_cube.jl:68-83,168-171,527): slot 4 of `correction` is read as a
 * per-cell mask; a cell whose entry is positive takes zero reconstruction offsets, a face
 * with such a cell on either side is solved by LLF (HLLD or HLL elsewhere), and the
 * admissibility check is on. The mask is the slot's content when the call is made: with
 * PMFMHD_RAD_TRACK_DENSITY as well (the reference accumulates the density increments into
 * the same slot during the launch) it is first copied into a context workspace, allocated on
 * the first such call. PMFMHD_RAD_GLOBAL_FALLBACK takes precedence over it, as CHECK == 3
 * does in the reference. GLM states only (the cube integrators do not run CT states):
 * PMFMHD_EUNSUPPORTED with ct_packed.
 */
int pmfmhd_step_radiation(pmfmhd_ctx* ctx, const pmfmhd_grid* g, const float* const U[9], float* const Unew[9],
                          float* ct_packed, float* correction, float dt, float ch, float decay, float drag_impulse,
                          int flags, void* stream);
/*
 * Fallback mask of the masked radiation step (`_radiation_fallback_mask_k!` and
 * `_radiation_expand_fallback_mask_k!`, radiation_coupling.jl:1536-1577): mask_out[c] = 1 if the
 * trial density of cell c or of one of its six face neighbours (periodic) is negative, or, with
 * mask_in non-null, if mask_in is positive there; 0 otherwise. mask_out must not overlap
 * trial_rho or mask_in. The reference's kernels need a cubic box; any periodic box is accepted
 * here (all-periodic boundaries required).
 */
int pmfmhd_radiation_fallback_mask(pmfmhd_ctx* ctx, const pmfmhd_grid* g, const float* trial_rho,
                                   const float* mask_in, float* mask_out, void* stream);
/*
 * In-place exact linear drag with velocity decay factor `decay` in [0, 1]
 * (`apply_linear_drag!`, drag.jl:78-117): m <- rho v0 + (m - rho v0) decay with
 * rho floored at smallr, E changed by the kinetic-energy change and floored at 1e-30.
 * energy_residual (n cells, nullable) Kahan-compensates E as `energy_compensation`.
 * Reads U[0..4] only.
 */
int pmfmhd_apply_linear_drag(pmfmhd_ctx* ctx, const pmfmhd_grid* g, float* const U[9], float decay,
                             const float target_velocity[3], float* energy_residual, void* stream);
/*
 * In-place exponential constant-force correction of a no-drag trial U given the state
 * before it (`apply_exponential_drag_increment!`, drag.jl:121-208). Reads old_U[0..3].
 */
int pmfmhd_apply_exponential_drag_increment(pmfmhd_ctx* ctx, const pmfmhd_grid* g, float* const U[9],
                                            const float* const old_U[9], float drag_impulse,
                                            const float target_velocity[3], void* stream);

/*
 * Max signal speed max over cells and axes of |v_d| + c_fast,d (timestep.jl:4-14,
 * `max_wavespeed!` :17-23). Blocking; *smax receives the host value.
 */
int pmfmhd_max_wavespeed(pmfmhd_ctx* ctx, const pmfmhd_grid* g, const float* const U[9], float* smax,
                         void* stream);
/* CFL step dt = cfl*dx/max(smax, eps) and smax (timestep.jl:37-41, `compute_dt!`). Blocking. */
int pmfmhd_compute_dt(pmfmhd_ctx* ctx, const pmfmhd_grid* g, const float* const U[9], float cfl, float* dt,
                      float* smax, void* stream);
/* Max signal speed of the state written by the last pmfmhd_step_glm / pmfmhd_step_ct on
 * this context (reduced on the device in that launch). Blocking. */
int pmfmhd_last_wavespeed(pmfmhd_ctx* ctx, float* smax, void* stream);

/* Max |div B| by BC-aware centred differences (diagnostics.jl:6-36). FP64 result. Blocking. */
int pmfmhd_max_divb(pmfmhd_ctx* ctx, const pmfmhd_grid* g, const float* const U[9], double* out, void* stream);
/* Max face divergence |sum_d (b_d[upper]-b_d[lower])|/dx of a CT face field (ct.jl:176-201). */
int pmfmhd_max_divb_face(pmfmhd_ctx* ctx, const pmfmhd_grid* g, const float* ct_packed, double* out,
                         void* stream);
/* FP64 volume integrals (mass, momx, momy, momz, energy, Bx, By, Bz) * dx^3
 * (diagnostics.jl:44-55, `conserved_totals`). Blocking. */
int pmfmhd_conserved_totals(pmfmhd_ctx* ctx, const pmfmhd_grid* g, const float* const U[9], double out[8],
                            void* stream);

/*
 * The same FP64 totals without a context and without allocating anything. No counterpart
 * in the reference. For callers that cannot call cudaMalloc (a host that owns the device
 * memory pool, a plugin inside another application, code that must not allocate between
 * steps): the scratch is a 4 MiB file-scope __device__ array of this library, held by every
 * GPU that loads it until exit. At most 2^24 cells (256^3); larger grids return
 * PMFMHD_ESHAPE. One partial sum per 256-cell block in a fixed order, so the result does not
 * depend on the SM count. Calls share the array: calls that overlap on the GPU race and
 * must be serialised. The first call in each CUDA context looks up the array's address and
 * caches it with the context's id; a context re-created later (cudaDeviceReset, or a host that
 * rebuilds its primary context) gets a fresh look-up on its first call, since the library's
 * module, and with it the array, may then sit elsewhere. Make the first call of a context
 * before any stream capture. Blocking.
 */
int pmfmhd_conserved_totals_noalloc(const pmfmhd_grid* g, const float* const U[9], double out[8], void* stream);

/*
 * CT initialisation from an EDGE-centred vector potential A (3 device arrays, Ax at
 * (i,j-1/2,k-1/2), Ay at (i-1/2,j,k-1/2), Az at (i-1/2,j-1/2,k)): faces = discrete curl,
 * cell B = face average, E adjusted to keep the thermal pressure, psi = 0, face remainders
 * zeroed (ct.jl:310-345 `ct_faces_from_potential!`, :205-236).
 */
int pmfmhd_ct_faces_from_potential(pmfmhd_ctx* ctx, const pmfmhd_grid* g, const float* const A[3],
                                   float* const U[9], float* ct_packed, void* stream);
/*
 * Install the face field the caller wrote into ct_packed slots 0-2: face remainders zeroed,
 * cell B = face average, E adjusted to keep the thermal pressure, psi = 0
 * (`_ct_install_faces!`, ct.jl:222-236).
 */
int pmfmhd_ct_install_faces(pmfmhd_ctx* ctx, const pmfmhd_grid* g, float* const U[9], float* ct_packed,
                            void* stream);

/*
 * nsteps GLM steps with a fixed dt/ch/decay, ping-ponging between U and scratch, recorded
 * once into a CUDA graph per (grid, buffers, nsteps) and replayed: the warm throughput
 * loop of scripts/benchmark.jl:53-62 (`advance()` repeated). After an even number of
 * steps the state is in U, after an odd number in scratch.
 */
int pmfmhd_run_glm(pmfmhd_ctx* ctx, const pmfmhd_grid* g, float* const U[9], float* const scratch[9],
                   int nsteps, float dt, float ch, float decay, float* const resid[7], void* stream);

/*
 * Batched form: many independent periodic boxes of uneven sizes advanced together.
 * Each box carries its own grid, buffers, solver and CFL settings; one pmfmhd_batch_step
 * advances every box by one step with its own device-computed dt (CFL on the box's
 * current state, ch = glm_ch_fac*smax, decay = exp(-glm_cr*ch*dt/dx), as `evolve!`,
 * driver.jl:48-71), using one persistent work-queued launch per solver family. Steps
 * are recorded into a CUDA graph on first use. No reference counterpart beyond
 * looping `evolve!` over boxes.
 */
typedef struct pmfmhd_box {
  pmfmhd_grid grid;
  float* U[9];
  float* scratch[9];
  float* ct_packed; /* NULL for GLM boxes; 21*nc floats for CT boxes */
  float* resid[7];  /* all NULL, or 7 remainder arrays (compensated update) */
  int32_t mhd_solver; /* 0 = GLM, 1 = CT */
  float cfl, glm_ch_fac, glm_cr;
} pmfmhd_box;
typedef struct pmfmhd_batch pmfmhd_batch;
int pmfmhd_batch_create(pmfmhd_ctx* ctx, const pmfmhd_box* boxes, int nbox, pmfmhd_batch** out);
int pmfmhd_batch_step(pmfmhd_batch* b, int nsteps, void* stream);
/* Per-box results after the last step: time advanced, current-state index (0: U, 1: scratch),
 * dt of the next step. Any pointer may be NULL. Blocking. */
int pmfmhd_batch_query(pmfmhd_batch* b, double* t, int32_t* parity, float* dt);
int pmfmhd_batch_destroy(pmfmhd_batch* b);

/* Tile autotuning: time the candidate tile shapes for this grid/solver on scratch copies
 * of U and remember the fastest in the context (used by every later step). Blocking. */
int pmfmhd_autotune(pmfmhd_ctx* ctx, const pmfmhd_grid* g, const float* const U[9], int mhd_solver,
                    int compensated, void* stream);

/*
 * pmfmhd_step_glm (plain update, MC-PLM with HLLD only) that also counts the HLLD single-star
 * degeneracy cases over every face of the grid once: out[0] = HLLD solves (faces not sent to
 * the LLF fallback), out[1] = single-star sides with |denK| < 1e-12 (the reference's degenerate
 * branch), out[2] = sides with 1e-12 <= |denK| < 1e-5 bn^2 (sent to the degenerate branch by
 * the relative tolerance only, i.e. the faces where the two tolerances give different fluxes).
 * The step is performed with g->hlld_dtol_rel as given. A diagnostic of the tolerance choice;
 * no counterpart in the reference. PMFMHD_EUNSUPPORTED for other reconstructions or solvers.
 * Blocking.
 */
int pmfmhd_step_glm_census(pmfmhd_ctx* ctx, const pmfmhd_grid* g, const float* const U[9], float* const Unew[9],
                           float dt, float ch, float decay, uint64_t out[3], void* stream);

/*
 * Test hook for the bounded TMA wait, normally 0. With polls > 0, every TMA-staged plane of
 * the steps enqueued afterwards on this context arms its mbarrier without issuing the copies
 * and gives up after `polls` polls: the wait runs out with nothing in flight, the status
 * becomes PMFMHD_ETIMEOUT and the step finishes by loading its planes straight from global
 * memory (its result is still the step's). polls = 0 restores normal staging.
 */
int pmfmhd_set_tma_stall(pmfmhd_ctx* ctx, int polls);

/* Device status of the steps enqueued on this context since the last clearing call:
 * PMFMHD_ETIMEOUT if a step kernel's bounded wait for a TMA plane load gave up, else
 * PMFMHD_OK. After a give-up the launch stops using its staging buffer (a late copy may still
 * land there) and loads every later plane straight from global memory, so the step still
 * completes with its own result; before exiting, each CTA gives the outstanding copy one more
 * bounded wait. clear != 0 resets the status. Blocking. */
int pmfmhd_status(pmfmhd_ctx* ctx, int clear, void* stream);

/* Pin (or query) the tile used for this grid/solver/mode on this context: `rows` owned rows
 * per CTA (an instantiated height: 5, 8, 9 or 13) and `planes` z-planes per CTA chunk. */
int pmfmhd_set_tile(pmfmhd_ctx* ctx, const pmfmhd_grid* g, int mhd_solver, int compensated, int rows, int planes);
int pmfmhd_get_tile(pmfmhd_ctx* ctx, const pmfmhd_grid* g, int mhd_solver, int compensated, int* rows,
                    int* planes);

/* ---- Terminal-regime induction (terminal_ct.jl) -------------------------------------- */
/* All on cubic periodic grids (PMFMHD_ESHAPE / PMFMHD_EUNSUPPORTED otherwise). */

/* Centred conservative Maxwell-stress force of B into F (`terminal_magnetic_force!`,
 * terminal_ct.jl:18-51,99-106). With P non-null the force is split (`..._split!`, :53-69,
 * :117-126): P = magnetic pressure -grad(B^2/2), F = the tension remainder. */
int pmfmhd_terminal_magnetic_force(pmfmhd_ctx* ctx, const pmfmhd_grid* g, const float* const B[3],
                                   float* const F[3], float* const P[3], void* stream);
/* Max terminal speed |v|, v = (F - c_p grad rho)/(max(rho, smallr) Gamma) capped at vcap
 * (`terminal_velocity_max!`, terminal_ct.jl:125-145,226-238). Reads U[0], U[5..7]. Blocking. */
int pmfmhd_terminal_velocity_max(pmfmhd_ctx* ctx, const pmfmhd_grid* g, const float* const U[9], float gamma_drag,
                                 float pressure_coeff, float vcap, double* vmax, void* stream);
/*
 * Terminal-regime SSPRK2 induction over dt (`terminal_ct_induction!`, terminal_ct.jl:502-575):
 * nsub = ceil(dt vmax / (cfl dx)) subcycles (PMFMHD_EINADMISSIBLE above max_subcycles), EMF
 * v x B from the terminal velocity recomputed at both stages, centred curl (GLM, ct_packed
 * NULL) or edge-averaged face curl (CT, faces Kahan-compensated through the packed
 * remainders when `compensate`), order-2 or order-4 dissipation with eta from vmax; E
 * follows the magnetic energy. Density and thermal energy are held. scratch (9 arrays) and
 * the CT workspace slots are overwritten. Outputs nsub, vmax, eta (nullable).
 */
int pmfmhd_terminal_ct_induction(pmfmhd_ctx* ctx, const pmfmhd_grid* g, float* const U[9], float* const scratch[9],
                                 float* ct_packed, float dt, float gamma_drag, float pressure_coeff, float cfl,
                                 float dissipation, int dissipation_order, float vcap, int max_subcycles,
                                 int compensate, int* nsub, double* vmax, double* eta, void* stream);
/* One compensated forward-Euler face update from the cell EMFs the caller left in the CT
 * slots ecx/ecy/ecz, then cell B = face average with E following and psi = 0
 * (`terminal_ct_euler_from_cell_emf!`, terminal_ct.jl:461-486). */
int pmfmhd_terminal_ct_euler_from_cell_emf(pmfmhd_ctx* ctx, const pmfmhd_grid* g, float* const U[9],
                                           float* ct_packed, float dt, void* stream);

/* ---- Initial conditions ------------------------------------------------------------- */

/* Mode realizations of the PMF generator (pmf.jl:193-203). The reference's `:legacy`
 * realization draws from Julia's MersenneTwister and is not provided. */
#define PMFMHD_PMF_HASH 1            /* :physical_hash */
#define PMFMHD_PMF_HASH_ZERO_PHASE 2 /* :physical_hash_zero_phase */

/* Arguments of `pmf_batchelor_field` (pmf.jl:300-317); "none" values as noted. */
typedef struct pmfmhd_pmf_params {
  int32_t nx, ny, nz;          /* nx even */
  int32_t realization;         /* PMFMHD_PMF_HASH or PMFMHD_PMF_HASH_ZERO_PHASE */
  int64_t seed;
  double box;                  /* box side L */
  double brms;                 /* target rms (> 0) */
  double realization_box;      /* <= 0: = box; realization_box / box must be an integer */
  double kcut;                 /* <= 0: pi * min(dims) / box */
  double kmin;                 /* >= 0 */
  double kmax;                 /* <= 0: no band limit */
  double energy_index;         /* 4: shell energy ~ k^4 */
  double cutoff_order;         /* 2 */
  int32_t curl_symbol;         /* 0: centred sin(k dx)/dx, 1: continuum k */
  int32_t curl_reference_n;    /* 0: none */
  int32_t fixed_mode_power;    /* rescale every mode to the analytic envelope */
  int32_t invariant_axis;      /* 0: none, 1..3: modes with k_axis != 0 removed */
  double preserve_low_kmax;    /* <= 0: none */
  double preserve_low_kcut;    /* <= 0: = kcut */
  int32_t normalization;       /* 0: auto, 1: total band rms, 2: reference (low) band rms */
  int32_t mode_lock_n;         /* 0: none */
  int32_t high_mode_lock_n;    /* 0: none */
  int32_t reserved;
  double minimum_cells_per_wavelength; /* <= 0: not enforced */
} pmfmhd_pmf_params;

/*
 * Non-helical Batchelor-spectrum magnetic field (`pmf_batchelor_field`, pmf.jl:300-591) into
 * three caller arrays of nx*ny*nz floats (x fastest): hashed vector-potential modes keyed
 * by physical mode number (pmf.jl:109-191), B = i s(k) x A(k) with the kcut taper, the
 * kmin/kmax band, optional centred-curl reference projection, mode locking, the preserved
 * low band and fixed mode power, then an inverse real FFT (cuFFT) and the rms
 * normalisation. stats (nullable): total brms, reference-band brms, normalisation brms,
 * kcut, kmax, high-source scale. Validation errors are PMFMHD_EINVAL / PMFMHD_ESHAPE, a zero
 * field PMFMHD_EINADMISSIBLE. Allocates transient workspace (about 5 floats per cell).
 */
int pmfmhd_pmf_batchelor_field(pmfmhd_ctx* ctx, const pmfmhd_pmf_params* p, float* const B[3], double stats[6],
                               void* stream);
/* dst (nx*ny*nz) = src (sx*sy*sz) repeated periodically; each tile extent must divide the
 * grid's (`_periodic_tile_field`, pmf.jl:226-237, used by `init_pmf_batchelor_tiled!`). */
int pmfmhd_periodic_tile(pmfmhd_ctx* ctx, const float* src, int sx, int sy, int sz, float* dst, int nx, int ny,
                         int nz, void* stream);
/* Uniform gas around the field in U[5..7] (`_install_pmf_field!`, pmf.jl:239-261):
 * rho = rho0, zero momentum, E = p0/(gamma-1) + |B|^2/2, psi = 0. */
int pmfmhd_pmf_install(pmfmhd_ctx* ctx, const pmfmhd_grid* g, float* const U[9], float rho0, float p0,
                       void* stream);
/*
 * Discretely divergence-free CT faces from the cell field U[5..7] (`ct_faces_from_cells!`,
 * ct.jl:246-308): FP64 cuFFT, projection onto tan(theta).b = 0, half-cell phase shift,
 * faces installed as by pmfmhd_ct_install_faces. stats (nullable): relative L2 change of the
 * cell field, magnetic energy ratio, max face div * dx / Brms. Allocates transient FP64
 * workspace (about 7 doubles per cell).
 */
int pmfmhd_ct_faces_from_cells(pmfmhd_ctx* ctx, const pmfmhd_grid* g, float* const U[9], float* ct_packed,
                               double stats[3], void* stream);

#ifdef __cplusplus
}
#endif
#endif /* PMFMHD_H */
