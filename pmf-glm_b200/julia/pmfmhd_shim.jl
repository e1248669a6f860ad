# Julia side of libpmfmhd.so: the ccall methods that route MHDKernels' CUDA step onto the
# library. Add to lib/MHDKernels/ext/MHDKernelsCUDAExt.jl (inside the extension module, where
# MHDKernels, CUDA and CUDABackend are in scope). The extension already has the seam:
# `_cube_launch!(::Val{:raw}, ::CUDABackend, ...)` (MHDKernelsCUDAExt.jl:22-26), which today
# raises "disabled". Only plain pointers, sizes and scalars cross the boundary
# (include/pmfmhd.h); the CuArrays stay owned by Julia.

const libpmfmhd = get(ENV, "PMFMHD_LIB", "libpmfmhd.so")

# HLLD single-star degeneracy tolerance (pmfmhd_grid.hlld_dtol_rel): 0 is the reference's own
# test |denK| < 1e-12 (glm_physics.jl:257); 1e-5 (the library's default) sends faces with
# |denK| < 1e-5 bn^2 to the degenerate branch.
const PMFMHD_HLLD_DTOL_REL = parse(Float32, get(ENV, "PMFMHD_HLLD_DTOL_REL", "1e-5"))

struct PmfGrid            # include/pmfmhd.h: pmfmhd_grid
    nx::Int32; ny::Int32; nz::Int32
    bc::NTuple{3,Int32}
    recon::Int32; riemann::Int32
    dx::Float32; gamma::Float32; smallr::Float32; pfl::Float32
    llf_dmin::Float32; llf_pmin::Float32
    hlld_dtol_rel::Float32
end
PmfGrid(s::MHDKernels.MHDState{Float32}) = PmfGrid(Int32.(s.dims)..., Int32.(MHDKernels.bc_codes(s)),
    Int32(MHDKernels.recon_code_of(s)), Int32(MHDKernels.riemann_code_of(s)),
    s.dx, s.γ, s.smallr, s.pfl, s.llf_dmin, s.llf_pmin, PMFMHD_HLLD_DTOL_REL)

const _pmf_ctx = Ref{Ptr{Cvoid}}(C_NULL)
function _pmf()                       # one library context per process/device
    if _pmf_ctx[] == C_NULL
        h = Ref{Ptr{Cvoid}}(C_NULL)
        rc = ccall((:pmfmhd_create, libpmfmhd), Cint, (Cint, Ptr{Ptr{Cvoid}}), CUDA.deviceid(), h)
        rc == 0 || error("pmfmhd_create: ", _pmf_err(rc))
        _pmf_ctx[] = h[]
    end
    _pmf_ctx[]
end
_pmf_err(rc) = unsafe_string(ccall((:pmfmhd_strerror, libpmfmhd), Cstring, (Cint,), rc))
_ptrs(t) = [pointer(a) for a in t]     # CuPtr{Float32} -> device addresses
_stream() = CUDA.stream().handle

# GLM: the drop-in for the fused cube launch (integrator_cube.jl:467-476)
function MHDKernels._cube_launch!(::Val{:raw}, ::CUDABackend, s::MHDKernels.MHDState{Float32},
                                  dt::Real, ch::Real, decay::Real)
    g = Ref(PmfGrid(s))
    rc = ccall((:pmfmhd_step_glm, libpmfmhd), Cint,
               (Ptr{Cvoid}, Ref{PmfGrid}, Ptr{CuPtr{Float32}}, Ptr{CuPtr{Float32}},
                Cfloat, Cfloat, Cfloat, Ptr{CuPtr{Float32}}, Ptr{Cvoid}),
               _pmf(), g, _ptrs(s.U), _ptrs(s.scratch), dt, ch, decay, C_NULL, _stream())
    rc == 0 || error("pmfmhd_step_glm: ", _pmf_err(rc))
    CUDA.synchronize()                 # the contract of _cube_launch!: return after completion
end
MHDKernels._cube_launch!(::Val{:auto}, be::CUDABackend, s::MHDKernels.MHDState{Float32}, dt::Real,
                         ch::Real, decay::Real) = MHDKernels._cube_launch!(Val(:raw), be, s, dt, ch, decay)

# CT: step!'s CT branch (driver.jl:22-27) = Godunov + ct_update!, one call
function pmf_step_ct!(s::MHDKernels.MHDState{Float32}, dt::Real; compensate::Bool=false)
    g = Ref(PmfGrid(s))
    rc = ccall((:pmfmhd_step_ct, libpmfmhd), Cint,
               (Ptr{Cvoid}, Ref{PmfGrid}, Ptr{CuPtr{Float32}}, Ptr{CuPtr{Float32}}, CuPtr{Float32},
                Cfloat, Ptr{CuPtr{Float32}}, Cint, Ptr{Cvoid}),
               _pmf(), g, _ptrs(s.U), _ptrs(s.scratch), pointer(s.ct.packed), dt, C_NULL,
               Cint(compensate), _stream())
    rc == 0 || error("pmfmhd_step_ct: ", _pmf_err(rc))
    s.U, s.scratch = s.scratch, s.U
    s
end

# Source-coupled drag step (drag.jl:162-178 -> step_ref_drag! / step_cube_drag!)
function MHDKernels.step_ref_drag!(s::MHDKernels.MHDState{Float32}, dt::Real; ch::Real, decay::Real,
                                   drag_impulse::Real, target_velocity=(0, 0, 0))
    v0 = Float32[target_velocity...]
    if MHDKernels.uses_ct(s)
        rc = ccall((:pmfmhd_step_ct_drag, libpmfmhd), Cint,
                   (Ptr{Cvoid}, Ref{PmfGrid}, Ptr{CuPtr{Float32}}, Ptr{CuPtr{Float32}}, CuPtr{Float32},
                    Cfloat, Cfloat, Ptr{Float32}, Ptr{Cvoid}),
                   _pmf(), Ref(PmfGrid(s)), _ptrs(s.U), _ptrs(s.scratch), pointer(s.ct.packed), dt,
                   drag_impulse, v0, _stream())
    else
        rc = ccall((:pmfmhd_step_glm_drag, libpmfmhd), Cint,
                   (Ptr{Cvoid}, Ref{PmfGrid}, Ptr{CuPtr{Float32}}, Ptr{CuPtr{Float32}},
                    Cfloat, Cfloat, Cfloat, Cfloat, Ptr{Float32}, Ptr{Cvoid}),
                   _pmf(), Ref(PmfGrid(s)), _ptrs(s.U), _ptrs(s.scratch), dt, ch, decay,
                   drag_impulse, v0, _stream())
    end
    rc == 0 || error("pmfmhd_step_*_drag: ", _pmf_err(rc))
    CUDA.synchronize()
    s.U, s.scratch = s.scratch, s.U
    s
end

# Radiation-coupled step (integrator_ref.jl:238-258): `correction` is the workspace's
# packed_psi_correction buffer as is (slot 0 = psi, 1-3 velocity corrections, 4-8 tracking)
function MHDKernels.step_ref_radiation!(s::MHDKernels.MHDState{Float32}, dt::Real; ch::Real, decay::Real,
                                        drag_impulse::Real, correction, track_density::Bool=true,
                                        track_magnetic::Bool=true, track_energy::Bool=true,
                                        robust_fallback::Bool=false)
    flags = Cint(track_density) | Cint(track_magnetic) << 1 | Cint(track_energy) << 2 |
            Cint(robust_fallback) << 4
    ctp = MHDKernels.uses_ct(s) ? pointer(s.ct.packed) : CuPtr{Float32}(0)
    rc = ccall((:pmfmhd_step_radiation, libpmfmhd), Cint,
               (Ptr{Cvoid}, Ref{PmfGrid}, Ptr{CuPtr{Float32}}, Ptr{CuPtr{Float32}}, CuPtr{Float32},
                CuPtr{Float32}, Cfloat, Cfloat, Cfloat, Cfloat, Cint, Ptr{Cvoid}),
               _pmf(), Ref(PmfGrid(s)), _ptrs(s.U), _ptrs(s.scratch), ctp, pointer(correction),
               dt, ch, decay, drag_impulse, flags, _stream())
    rc == 0 || error("pmfmhd_step_radiation: ", _pmf_err(rc))
    CUDA.synchronize()
    s.U, s.scratch = s.scratch, s.U
    s
end
# step_cube_radiation! (integrator_cube.jl:504-540; GLM states only, as in the reference): the
# same call with check_admissibility (bit 3), global_fallback (bit 5) and the masked fallback
# (bit 6, `fallback=true`: slot 4 of `correction` is the per-cell mask, e.g. from
# pmf_radiation_fallback_mask!)
function MHDKernels.step_cube_radiation!(s::MHDKernels.MHDState{Float32}, dt::Real; ch::Real, decay::Real,
                                         drag_impulse::Real, correction, track_density::Bool=true,
                                         track_magnetic::Bool=true, track_energy::Bool=true,
                                         check_admissibility::Bool=false, fallback::Bool=false,
                                         global_fallback::Bool=false, robust_fallback::Bool=false)
    flags = Cint(track_density) | Cint(track_magnetic) << 1 | Cint(track_energy) << 2 |
            Cint(check_admissibility) << 3 | Cint(robust_fallback) << 4 | Cint(global_fallback) << 5 |
            Cint(fallback) << 6
    rc = ccall((:pmfmhd_step_radiation, libpmfmhd), Cint,
               (Ptr{Cvoid}, Ref{PmfGrid}, Ptr{CuPtr{Float32}}, Ptr{CuPtr{Float32}}, CuPtr{Float32},
                CuPtr{Float32}, Cfloat, Cfloat, Cfloat, Cfloat, Cint, Ptr{Cvoid}),
               _pmf(), Ref(PmfGrid(s)), _ptrs(s.U), _ptrs(s.scratch), CuPtr{Float32}(0), pointer(correction),
               dt, ch, decay, drag_impulse, flags, _stream())
    rc == 0 || error("pmfmhd_step_radiation: ", _pmf_err(rc))
    CUDA.synchronize()
    s.U, s.scratch = s.scratch, s.U
    s
end

# The masked fallback's mask (radiation_coupling.jl:1536-1593) into `mask` (ncells Float32 on
# the device): from the trial density, or expanded from `mask_in` as well
function pmf_radiation_fallback_mask!(mask, s::MHDKernels.MHDState{Float32}, trial_rho; mask_in=nothing)
    mp = mask_in === nothing ? CuPtr{Float32}(0) : pointer(mask_in)
    rc = ccall((:pmfmhd_radiation_fallback_mask, libpmfmhd), Cint,
               (Ptr{Cvoid}, Ref{PmfGrid}, CuPtr{Float32}, CuPtr{Float32}, CuPtr{Float32}, Ptr{Cvoid}),
               _pmf(), Ref(PmfGrid(s)), pointer(trial_rho), mp, pointer(mask), _stream())
    rc == 0 || error("pmfmhd_radiation_fallback_mask: ", _pmf_err(rc))
    mask
end

# CFL reduction (timestep.jl:37-41) without the N^3 work array or a host maximum()
function pmf_compute_dt(s::MHDKernels.MHDState{Float32}; cfl::Real=0.4)
    dt = Ref{Float32}(); smax = Ref{Float32}()
    rc = ccall((:pmfmhd_compute_dt, libpmfmhd), Cint,
               (Ptr{Cvoid}, Ref{PmfGrid}, Ptr{CuPtr{Float32}}, Cfloat, Ref{Float32}, Ref{Float32}, Ptr{Cvoid}),
               _pmf(), Ref(PmfGrid(s)), _ptrs(s.U), cfl, dt, smax, _stream())
    rc == 0 || error("pmfmhd_compute_dt: ", _pmf_err(rc))
    dt[], smax[]
end

# Device status of the steps so far (0, or the PMFMHD_ETIMEOUT code when a bounded TMA wait
# gave up; the step then finished from global memory)
pmf_status(; clear::Bool=true) = ccall((:pmfmhd_status, libpmfmhd), Cint, (Ptr{Cvoid}, Cint, Ptr{Cvoid}),
                                       _pmf(), Cint(clear), _stream())
