"""Host-side mirror of MHDKernels' step API over libpmfmhd.so (ctypes; torch owns memory).

The names, arguments and error behaviour follow lib/MHDKernels/src: ``allocate_state``
(state.jl:123-141), ``step`` / ``step_cube`` / ``step_ref`` (driver.jl:20-37,
integrator_cube.jl:455-463, integrator_ref.jl:210-220), ``evolve`` (driver.jl:48-71),
``compute_dt`` / ``max_wavespeed`` (timestep.jl:17-46), ``max_divb`` /
``conserved_totals`` (diagnostics.jl:22-55), ``max_divb_face`` / ``ct_faces_from_potential``
/ ``ct_faces_from_cells`` (ct.jl:187-345), the drag steps and operators of drag.jl
(``step_drag_godunov``, ``step_ref_drag`` / ``step_cube_drag``, ``apply_linear_drag``,
``apply_exponential_drag_increment``, ``step_drag_strang``, ``step_drag_exponential``,
``DragRegimeController`` / ``update_drag_regime``). Errors raise ``PMFMHDError`` where the
reference calls ``error(...)``. Every step runs the sm_100a CUDA library; there is no CPU
path, and a missing library raises at import of the first call.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
# PMFMHD_LIB overrides the library path (the same variable the Julia shim reads)
LIB_PATH = os.environ.get("PMFMHD_LIB", os.path.join(HERE, "libpmfmhd.so"))

GLM_CR = 0.18  # driver.jl:8
NVAR = 9
RECON = {"plm": 0, "ppm": 1, "plm_minmod": 2}
RIEMANN = {"hlld": 0, "hll": 1, "llf": 2}
BC = {"periodic": 0, "outflow": 1, "reflecting": 2}
CT_NSLOT = 21
FLOAT32_EPS = float(np.finfo(np.float32).eps)
# HLLD single-star degeneracy tolerance (pmfmhd_grid.hlld_dtol_rel): the degenerate branch is
# taken when |denK| < max(1e-12, dtol_rel * bn^2). 0.0 is the reference's own test
# |denK| < 1e-12 (glm_physics.jl:257); 1e-5, the default here, is the relative test.
HLLD_DTOL_REFERENCE = 0.0
HLLD_DTOL_RELATIVE = 1e-5


class PMFMHDError(RuntimeError):
    pass


class Grid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
                ("bc", ctypes.c_int32 * 3), ("recon", ctypes.c_int32), ("riemann", ctypes.c_int32),
                ("dx", ctypes.c_float), ("gamma", ctypes.c_float), ("smallr", ctypes.c_float),
                ("pfl", ctypes.c_float), ("llf_dmin", ctypes.c_float), ("llf_pmin", ctypes.c_float),
                ("hlld_dtol_rel", ctypes.c_float)]


class Box(ctypes.Structure):
    _fields_ = [("grid", Grid), ("U", ctypes.c_void_p * 9), ("scratch", ctypes.c_void_p * 9),
                ("ct_packed", ctypes.c_void_p), ("resid", ctypes.c_void_p * 7), ("mhd_solver", ctypes.c_int32),
                ("cfl", ctypes.c_float), ("glm_ch_fac", ctypes.c_float), ("glm_cr", ctypes.c_float)]


# Exported symbols and their signatures (include/pmfmhd.h).
_VP = ctypes.c_void_p
_P9 = ctypes.c_void_p * 9
_P7 = ctypes.c_void_p * 7
_P3 = ctypes.c_void_p * 3
_GP = ctypes.POINTER(Grid)
_F3P = ctypes.POINTER(ctypes.c_float)  # const float[3], nullable


class PmfParams(ctypes.Structure):
    """pmfmhd_pmf_params (include/pmfmhd.h)."""
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
                ("realization", ctypes.c_int32), ("seed", ctypes.c_int64), ("box", ctypes.c_double),
                ("brms", ctypes.c_double), ("realization_box", ctypes.c_double), ("kcut", ctypes.c_double),
                ("kmin", ctypes.c_double), ("kmax", ctypes.c_double), ("energy_index", ctypes.c_double),
                ("cutoff_order", ctypes.c_double), ("curl_symbol", ctypes.c_int32),
                ("curl_reference_n", ctypes.c_int32), ("fixed_mode_power", ctypes.c_int32),
                ("invariant_axis", ctypes.c_int32), ("preserve_low_kmax", ctypes.c_double),
                ("preserve_low_kcut", ctypes.c_double), ("normalization", ctypes.c_int32),
                ("mode_lock_n", ctypes.c_int32), ("high_mode_lock_n", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("minimum_cells_per_wavelength", ctypes.c_double)]

SIGNATURES = {
    "pmfmhd_version": ([], ctypes.c_int),
    "pmfmhd_strerror": ([ctypes.c_int], ctypes.c_char_p),
    "pmfmhd_last_cuda_error": ([], ctypes.c_char_p),
    "pmfmhd_create": ([ctypes.c_int, ctypes.POINTER(_VP)], ctypes.c_int),
    "pmfmhd_destroy": ([_VP], ctypes.c_int),
    "pmfmhd_step_glm": ([_VP, _GP, _P9, _P9, ctypes.c_float, ctypes.c_float, ctypes.c_float, _VP, _VP], ctypes.c_int),
    "pmfmhd_step_glm_host": ([_VP, _GP, _P9, _P9, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_int, _VP],
                             ctypes.c_int),
    "pmfmhd_step_ct": ([_VP, _GP, _P9, _P9, _VP, ctypes.c_float, _VP, ctypes.c_int, _VP], ctypes.c_int),
    "pmfmhd_step_glm_drag": ([_VP, _GP, _P9, _P9, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                              _F3P, _VP], ctypes.c_int),
    "pmfmhd_step_ct_drag": ([_VP, _GP, _P9, _P9, _VP, ctypes.c_float, ctypes.c_float, _F3P, _VP], ctypes.c_int),
    "pmfmhd_step_radiation": ([_VP, _GP, _P9, _P9, _VP, _VP, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                               ctypes.c_float, ctypes.c_int, _VP], ctypes.c_int),
    "pmfmhd_radiation_fallback_mask": ([_VP, _GP, _VP, _VP, _VP, _VP], ctypes.c_int),
    "pmfmhd_ct_install_faces": ([_VP, _GP, _P9, _VP, _VP], ctypes.c_int),
    "pmfmhd_terminal_magnetic_force": ([_VP, _GP, _P3, _P3, _VP, _VP], ctypes.c_int),
    "pmfmhd_terminal_velocity_max": ([_VP, _GP, _P9, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                      ctypes.POINTER(ctypes.c_double), _VP], ctypes.c_int),
    "pmfmhd_terminal_ct_induction": ([_VP, _GP, _P9, _P9, _VP, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                      ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_float, ctypes.c_int,
                                      ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double),
                                      ctypes.POINTER(ctypes.c_double), _VP], ctypes.c_int),
    "pmfmhd_terminal_ct_euler_from_cell_emf": ([_VP, _GP, _P9, _VP, ctypes.c_float, _VP], ctypes.c_int),
    "pmfmhd_pmf_batchelor_field": ([_VP, ctypes.POINTER(PmfParams), _P3, ctypes.c_double * 6, _VP], ctypes.c_int),
    "pmfmhd_pmf_install": ([_VP, _GP, _P9, ctypes.c_float, ctypes.c_float, _VP], ctypes.c_int),
    "pmfmhd_periodic_tile": ([_VP, _VP, ctypes.c_int, ctypes.c_int, ctypes.c_int, _VP, ctypes.c_int, ctypes.c_int,
                              ctypes.c_int, _VP], ctypes.c_int),
    "pmfmhd_ct_faces_from_cells": ([_VP, _GP, _P9, _VP, ctypes.c_double * 3, _VP], ctypes.c_int),
    "pmfmhd_apply_linear_drag": ([_VP, _GP, _P9, ctypes.c_float, _F3P, _VP, _VP], ctypes.c_int),
    "pmfmhd_apply_exponential_drag_increment": ([_VP, _GP, _P9, _P9, ctypes.c_float, _F3P, _VP], ctypes.c_int),
    "pmfmhd_max_wavespeed": ([_VP, _GP, _P9, ctypes.POINTER(ctypes.c_float), _VP], ctypes.c_int),
    "pmfmhd_compute_dt": ([_VP, _GP, _P9, ctypes.c_float, ctypes.POINTER(ctypes.c_float),
                           ctypes.POINTER(ctypes.c_float), _VP], ctypes.c_int),
    "pmfmhd_last_wavespeed": ([_VP, ctypes.POINTER(ctypes.c_float), _VP], ctypes.c_int),
    "pmfmhd_max_divb": ([_VP, _GP, _P9, ctypes.POINTER(ctypes.c_double), _VP], ctypes.c_int),
    "pmfmhd_max_divb_face": ([_VP, _GP, _VP, ctypes.POINTER(ctypes.c_double), _VP], ctypes.c_int),
    "pmfmhd_conserved_totals": ([_VP, _GP, _P9, ctypes.c_double * 8, _VP], ctypes.c_int),
    "pmfmhd_conserved_totals_noalloc": ([_GP, _P9, ctypes.c_double * 8, _VP], ctypes.c_int),
    "pmfmhd_ct_faces_from_potential": ([_VP, _GP, _P3, _P9, _VP, _VP], ctypes.c_int),
    "pmfmhd_run_glm": ([_VP, _GP, _P9, _P9, ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_float, _VP, _VP],
                       ctypes.c_int),
    "pmfmhd_batch_create": ([_VP, ctypes.POINTER(Box), ctypes.c_int, ctypes.POINTER(_VP)], ctypes.c_int),
    "pmfmhd_batch_step": ([_VP, ctypes.c_int, _VP], ctypes.c_int),
    "pmfmhd_batch_query": ([_VP, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int32),
                            ctypes.POINTER(ctypes.c_float)], ctypes.c_int),
    "pmfmhd_batch_destroy": ([_VP], ctypes.c_int),
    "pmfmhd_autotune": ([_VP, _GP, _P9, ctypes.c_int, ctypes.c_int, _VP], ctypes.c_int),
    "pmfmhd_status": ([_VP, ctypes.c_int, _VP], ctypes.c_int),
    "pmfmhd_step_glm_census": ([_VP, _GP, _P9, _P9, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                ctypes.c_uint64 * 3, _VP], ctypes.c_int),
    "pmfmhd_set_tma_stall": ([_VP, ctypes.c_int], ctypes.c_int),
    "pmfmhd_set_tile": ([_VP, _GP, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "pmfmhd_get_tile": ([_VP, _GP, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                         ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
}

_lib = None
_ctx = {}


def lib():
    """Load libpmfmhd.so; raise if it has not been built (there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise PMFMHDError(f"libpmfmhd.so not built at {LIB_PATH}; run `make -C {HERE}`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (argtypes, restype) in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = argtypes
            f.restype = restype
        _lib = L
    return _lib


def _check(rc, what):
    if rc != 0:
        L = lib()
        msg = L.pmfmhd_strerror(rc).decode()
        cuda = L.pmfmhd_last_cuda_error().decode()
        raise PMFMHDError(f"{what}: {msg} (code {rc})" + (f": {cuda}" if cuda and rc == -3 else ""))


def context(device: Optional[int] = None):
    """Per-device library context (reduction workspace, tile table, cached graphs)."""
    if device is None:
        device = torch.cuda.current_device()
    if device not in _ctx:
        if not torch.cuda.is_available():
            raise PMFMHDError("no CUDA device: libpmfmhd needs an sm_100a GPU")
        h = _VP()
        with torch.cuda.device(device):
            _check(lib().pmfmhd_create(device, ctypes.byref(h)), "pmfmhd_create")
        _ctx[device] = h
    return _ctx[device]


def _stream():
    return _VP(torch.cuda.current_stream().cuda_stream)


def _p9(ts) -> "ctypes.Array":
    return _P9(*[t.data_ptr() for t in ts])


@dataclass
class CTState:
    """Reference CTState (state.jl:44-58): one packed buffer of 21 slots of ncells."""
    packed: torch.Tensor
    nc: int

    def slot(self, q: int) -> torch.Tensor:
        return self.packed[q * self.nc:(q + 1) * self.nc]

    @property
    def bxf(self): return self.slot(0)
    @property
    def byf(self): return self.slot(1)
    @property
    def bzf(self): return self.slot(2)
    @property
    def rbx(self): return self.slot(18)
    @property
    def rby(self): return self.slot(19)
    @property
    def rbz(self): return self.slot(20)


@dataclass
class MHDState:
    U: list
    scratch: list
    dims: tuple
    dx: float
    gamma: float
    smallr: float
    pfl: float
    llf_dmin: float
    llf_pmin: float
    riemann: str
    recon: str
    bcs: tuple
    device: int
    ct: Optional[CTState] = None
    resid: Optional[list] = None
    grid: Grid = field(default=None, repr=False)

    @property
    def nc(self):
        return int(np.prod(self.dims))

    def uses_ct(self):
        return self.ct is not None

    def mhd_solver(self):
        return "ct" if self.ct is not None else "glm"


def uses_ct(s: MHDState) -> bool:
    return s.ct is not None


def allocate_state(dims: Sequence[int], dx: float, gamma: float = 5 / 3, smallr: float = 1e-6, pfl: float = 1e-7,
                   llf_dmin: float = 1e-4, llf_pmin: float = 0.0, use_hlld: bool = True, riemann=None,
                   bc: str = "periodic", bcs=None, recon: str = "plm", mhd_solver: str = "glm",
                   compensated: bool = False, device: Optional[int] = None,
                   hlld_dtol_rel: float = HLLD_DTOL_RELATIVE) -> MHDState:
    """Zero-filled FP32 state on the GPU (state.jl:123-141). ``compensated`` adds the seven
    Kahan remainder arrays of the compensated update (momentum, E, B). ``hlld_dtol_rel`` is
    the HLLD degeneracy tolerance (HLLD_DTOL_REFERENCE for the reference's own test)."""
    if not (np.isfinite(hlld_dtol_rel) and hlld_dtol_rel >= 0):
        raise PMFMHDError("hlld_dtol_rel must be finite and non-negative")
    if mhd_solver not in ("glm", "ct"):
        raise PMFMHDError(f"unknown mhd_solver :{mhd_solver} (have :glm, :ct)")
    bcs = tuple(bcs) if bcs is not None else (bc, bc, bc)
    for b in bcs:
        if b not in BC:
            raise PMFMHDError(f"unknown BC :{b} (have :periodic, :outflow, :reflecting)")
    if mhd_solver == "ct" and any(b != "periodic" for b in bcs):
        raise PMFMHDError(f"mhd_solver=:ct requires all-periodic boundaries (bcs={bcs}); "
                          "constrained transport is periodic-only")
    rsym = riemann if riemann is not None else ("hlld" if use_hlld else "llf")
    if rsym not in RIEMANN:
        raise PMFMHDError(f"unknown MHD riemann :{rsym} (have :hlld, :hll, :llf)")
    if recon not in RECON:
        raise PMFMHDError(f"unknown recon :{recon} (have :plm, :plm_minmod, :ppm)")
    if device is None:
        device = torch.cuda.current_device()
    dims = tuple(int(d) for d in dims)
    nc = int(np.prod(dims))
    dev = torch.device("cuda", device)
    U = [torch.zeros(nc, dtype=torch.float32, device=dev) for _ in range(NVAR)]
    sc = [torch.zeros(nc, dtype=torch.float32, device=dev) for _ in range(NVAR)]
    ct = CTState(torch.zeros(CT_NSLOT * nc, dtype=torch.float32, device=dev), nc) if mhd_solver == "ct" else None
    resid = [torch.zeros(nc, dtype=torch.float32, device=dev) for _ in range(7)] if compensated else None
    f32 = lambda v: float(np.float32(v))
    s = MHDState(U, sc, dims, f32(dx), f32(gamma), f32(smallr), f32(pfl), f32(llf_dmin), f32(llf_pmin), rsym, recon,
                 bcs, device, ct, resid)
    s.grid = Grid(dims[0], dims[1], dims[2], (ctypes.c_int32 * 3)(*[BC[b] for b in bcs]), RECON[recon],
                  RIEMANN[rsym], s.dx, s.gamma, s.smallr, s.pfl, s.llf_dmin, s.llf_pmin, f32(hlld_dtol_rel))
    return s


def set_fields(s: MHDState, U_host) -> MHDState:
    """Copy a host ``(9, nc)`` conserved array into the state."""
    U_host = np.ascontiguousarray(np.asarray(U_host, dtype=np.float32).reshape(NVAR, s.nc))
    for v in range(NVAR):
        s.U[v].copy_(torch.from_numpy(U_host[v]))
    return s


def fields_to_host(s: MHDState) -> np.ndarray:
    """``(9, nc)`` host copy of the conserved fields (state.jl:143-144)."""
    return torch.stack(s.U).cpu().numpy()


def _resid_arg(s: MHDState):
    return _P7(*[t.data_ptr() for t in s.resid]) if s.resid is not None else None


def step_cube(s: MHDState, dt: float, ch: float, decay: float) -> MHDState:
    """One GLM step into the scratch set, then swap (integrator_cube.jl:455-463)."""
    if uses_ct(s):
        raise PMFMHDError("step_cube!: CT is implemented on the :ref integrator only "
                          "(mhd_solver=:ct states cannot use the :cube integrators)")
    _check(lib().pmfmhd_step_glm(context(s.device), ctypes.byref(s.grid), _p9(s.U), _p9(s.scratch), float(dt),
                                 float(ch), float(decay), _resid_arg(s), _stream()), "step_cube!")
    s.U, s.scratch = s.scratch, s.U
    return s


def step_cube_host(s: MHDState, U_host: torch.Tensor, Unew_host: torch.Tensor, dt: float, ch: float, decay: float,
                   nchunks: int = 16) -> None:
    """The GLM step on host (9, nc) float32 tensors (pinned for PCIe/compute overlap) with the
    grid and parameters of ``s`` (pmfmhd_step_glm_host); ``s``'s device fields are not used."""
    for t in (U_host, Unew_host):
        if t.device.type != "cpu" or t.dtype != torch.float32 or tuple(t.shape) != (9, s.nc) or not t.is_contiguous():
            raise PMFMHDError("host state must be a contiguous float32 CPU tensor of shape (9, ncells)")
    _check(lib().pmfmhd_step_glm_host(context(s.device), ctypes.byref(s.grid), _p9(U_host), _p9(Unew_host), float(dt),
                                      float(ch), float(decay), int(nchunks), _stream()), "step_cube_host")


def step_ref(s: MHDState, dt: float, ch: float, decay: float, compensate_faces: bool = False) -> MHDState:
    """integrator_ref.jl:210-220 (+ ct_update!): the same fused kernel; CT states run the
    Godunov stage and the CT face update."""
    if uses_ct(s):
        _check(lib().pmfmhd_step_ct(context(s.device), ctypes.byref(s.grid), _p9(s.U), _p9(s.scratch),
                                    s.ct.packed.data_ptr(), float(dt), _resid_arg(s), int(compensate_faces),
                                    _stream()), "step_ref!")
        s.U, s.scratch = s.scratch, s.U
        return s
    return step_cube(s, dt, ch, decay)


def step(s: MHDState, dt: float, ch: Optional[float] = None, glm_cr: float = GLM_CR,
         integrator: str = "cube") -> MHDState:
    """driver.jl:20-37. CT states ignore ``ch``/``glm_cr``."""
    if integrator not in ("ref", "cube"):
        raise PMFMHDError(f"unknown integrator :{integrator} (have :ref, :cube)")
    if uses_ct(s):
        if integrator != "ref":
            raise PMFMHDError("step!: CT is implemented on the :ref integrator only "
                              "(mhd_solver=:ct states cannot use the :cube integrators)")
        return step_ref(s, dt, 0.0, 1.0)
    if ch is None:
        raise PMFMHDError("step! needs the GLM cleaning speed `ch` (GLM states)")
    T = np.float32
    decay = float(np.exp(T(T(-T(glm_cr) * T(ch) * T(dt)) / T(s.dx))))
    return step_cube(s, dt, ch, decay)


# ---- source-coupled drag (lib/MHDKernels/src/drag.jl) ---------------------------------------

def _target(v):
    v = tuple(float(x) for x in v)
    if len(v) != 3:
        raise PMFMHDError("target_velocity must have three components")
    return (ctypes.c_float * 3)(*v)


def _check_impulse(q):
    if not (np.isfinite(q) and q >= 0):
        raise PMFMHDError("drag impulse must be finite and non-negative")


def step_ref_drag(s: MHDState, dt: float, ch: float, decay: float, drag_impulse: float,
                  target_velocity=(0.0, 0.0, 0.0)) -> MHDState:
    """integrator_ref.jl:222-234: the fused step with the drag face prediction and the drag
    corrector (CT states then run ct_update! without face compensation)."""
    _check_impulse(drag_impulse)
    v0 = _target(target_velocity)
    if uses_ct(s):
        _check(lib().pmfmhd_step_ct_drag(context(s.device), ctypes.byref(s.grid), _p9(s.U), _p9(s.scratch),
                                         s.ct.packed.data_ptr(), float(dt), float(drag_impulse), v0, _stream()),
               "step_ref_drag!")
    else:
        _check(lib().pmfmhd_step_glm_drag(context(s.device), ctypes.byref(s.grid), _p9(s.U), _p9(s.scratch),
                                          float(dt), float(ch), float(decay), float(drag_impulse), v0, _stream()),
               "step_ref_drag!")
    s.U, s.scratch = s.scratch, s.U
    return s


def step_cube_drag(s: MHDState, dt: float, ch: float, decay: float, drag_impulse: float,
                   target_velocity=(0.0, 0.0, 0.0)) -> MHDState:
    """integrator_cube.jl:478-490: GLM states only, target at rest (the CMB frame). The
    cubic-grid and N % 4 conditions of the reference's 4^3 cube do not apply to this kernel."""
    if uses_ct(s):
        raise PMFMHDError("step_cube_drag!: CT is implemented on the :ref integrator only "
                          "(mhd_solver=:ct states cannot use the :cube integrators)")
    if any(float(v) != 0.0 for v in target_velocity):
        raise PMFMHDError("step_cube_drag! is specialized for Compton drag in the CMB frame; "
                          "use integrator=:ref for a moving target")
    return step_ref_drag(s, dt, ch, decay, drag_impulse)


def step_drag_godunov(s: MHDState, dt: float, drag_impulse: float, ch: float, glm_cr: float = GLM_CR,
                      integrator: str = "cube", target_velocity=(0.0, 0.0, 0.0)) -> MHDState:
    """drag.jl:162-178: one source-aware Godunov step; decay = exp(-cr*ch*dt/dx) in FP32."""
    _check_impulse(drag_impulse)
    T = np.float32
    decay = float(np.exp(T(T(-T(glm_cr) * T(ch) * T(dt)) / T(s.dx))))
    if integrator == "ref":
        return step_ref_drag(s, dt, ch, decay, drag_impulse, target_velocity)
    if integrator == "cube":
        return step_cube_drag(s, dt, ch, decay, drag_impulse, target_velocity)
    raise PMFMHDError(f"unknown integrator :{integrator} (have :ref, :cube)")


RAD_TRACK_DENSITY, RAD_TRACK_MAGNETIC, RAD_TRACK_ENERGY = 1, 2, 4
RAD_CHECK_ADMISSIBILITY, RAD_ROBUST_FALLBACK, RAD_GLOBAL_FALLBACK, RAD_MASKED_FALLBACK = 8, 16, 32, 64


def allocate_radiation_correction(s: MHDState) -> torch.Tensor:
    """A zeroed packed correction buffer (9*nc floats) with slot 0 set to the state's psi,
    the layout of the reference's ``packed_psi_correction`` (radiation_coupling.jl:207-214)."""
    corr = torch.zeros(9 * s.nc, dtype=torch.float32, device=s.U[0].device)
    corr[: s.nc].copy_(s.U[8])
    return corr


def _step_radiation(s, dt, ch, decay, drag_impulse, correction, flags, what):
    _check_impulse(drag_impulse)
    if correction.numel() != 9 * s.nc or correction.dtype != torch.float32 or not correction.is_contiguous():
        raise PMFMHDError(f"{what}: correction must be a contiguous float32 buffer of 9*ncells values")
    ct = s.ct.packed.data_ptr() if uses_ct(s) else None
    _check(lib().pmfmhd_step_radiation(context(s.device), ctypes.byref(s.grid), _p9(s.U), _p9(s.scratch), ct,
                                       correction.data_ptr(), float(dt), float(ch), float(decay),
                                       float(drag_impulse), int(flags), _stream()), what)
    s.U, s.scratch = s.scratch, s.U
    return s


def step_ref_radiation(s: MHDState, dt: float, ch: float, decay: float, drag_impulse: float, correction,
                       track_density: bool = True, track_magnetic: bool = True, track_energy: bool = True,
                       robust_fallback: bool = False) -> MHDState:
    """integrator_ref.jl:238-258: the drag step whose face states carry the velocity
    corrections of ``correction`` (slot 0 = psi), with the tracked density increment and
    the Kahan remainders of B and E kept in it; CT faces are compensated with
    ``track_magnetic``. ``robust_fallback`` runs minmod PLM with HLL."""
    flags = ((RAD_TRACK_DENSITY if track_density else 0) | (RAD_TRACK_MAGNETIC if track_magnetic else 0)
             | (RAD_TRACK_ENERGY if track_energy else 0) | (RAD_ROBUST_FALLBACK if robust_fallback else 0))
    return _step_radiation(s, dt, ch, decay, drag_impulse, correction, flags, "step_ref_radiation!")


def step_cube_radiation(s: MHDState, dt: float, ch: float, decay: float, drag_impulse: float, correction,
                        track_density: bool = True, track_magnetic: bool = True, track_energy: bool = True,
                        check_admissibility: bool = False, fallback: bool = False, global_fallback: bool = False,
                        robust_fallback: bool = False) -> MHDState:
    """integrator_cube.jl:504-540 (GLM states): as step_ref_radiation, plus the admissibility
    flag (rejected cells get density -max(|rho|, max(smallr, llf_dmin))), the global
    fallback (piecewise-constant states with LLF, the cube kernel's CHECK == 3) and the
    masked fallback (``fallback=True``, CHECK == 2): slot 4 of ``correction`` is a per-cell
    mask (see ``radiation_fallback_mask``); masked cells take piecewise-constant states, every
    face touching one is solved by LLF, and the admissibility flag is on. The mask is read as
    it is when the call is made, before this step's density increments land in the same slot.
    ``global_fallback`` takes precedence over ``fallback``; ``robust_fallback`` with
    ``fallback`` runs minmod PLM / HLL with the masked cells and faces as above."""
    if uses_ct(s):
        raise PMFMHDError("step_cube_radiation!: CT is implemented on the :ref integrator only "
                          "(mhd_solver=:ct states cannot use the :cube integrators)")
    flags = ((RAD_TRACK_DENSITY if track_density else 0) | (RAD_TRACK_MAGNETIC if track_magnetic else 0)
             | (RAD_TRACK_ENERGY if track_energy else 0) | (RAD_CHECK_ADMISSIBILITY if check_admissibility else 0)
             | (RAD_ROBUST_FALLBACK if robust_fallback else 0) | (RAD_GLOBAL_FALLBACK if global_fallback else 0)
             | (RAD_MASKED_FALLBACK if fallback else 0))
    return _step_radiation(s, dt, ch, decay, drag_impulse, correction, flags, "step_cube_radiation!")


def radiation_fallback_mask(s: MHDState, trial_rho: torch.Tensor, mask_in: Optional[torch.Tensor] = None,
                            out: Optional[torch.Tensor] = None) -> torch.Tensor:
    """The masked fallback's mask (radiation_coupling.jl:1536-1577): 1 where the trial density
    of a cell or of one of its six periodic face neighbours is negative, or, with ``mask_in``
    (``_radiation_expand_fallback_mask!``), where that mask is positive there as well; 0
    elsewhere. Returns ``out`` (a new tensor if None), which must not overlap the inputs. To
    use it in a step, write it into slot 4 of the correction buffer."""
    nc = s.nc
    for t, what in ((trial_rho, "trial_rho"), (mask_in, "mask_in")):
        if t is not None and (t.numel() != nc or t.dtype != torch.float32 or not t.is_contiguous()):
            raise PMFMHDError(f"radiation_fallback_mask: {what} must be a contiguous float32 field of ncells values")
    if out is None:
        out = torch.empty(nc, dtype=torch.float32, device=trial_rho.device)
    elif out.numel() != nc or out.dtype != torch.float32 or not out.is_contiguous():
        raise PMFMHDError("radiation_fallback_mask: out must be a contiguous float32 field of ncells values")
    _check(lib().pmfmhd_radiation_fallback_mask(context(s.device), ctypes.byref(s.grid), trial_rho.data_ptr(),
                                                mask_in.data_ptr() if mask_in is not None else None,
                                                out.data_ptr(), _stream()), "radiation_fallback_mask")
    return out


def apply_linear_drag(s: MHDState, decay: float, target_velocity=(0.0, 0.0, 0.0),
                      energy_compensation: Optional[torch.Tensor] = None) -> MHDState:
    """drag.jl:78-117: exact linear drag with velocity decay factor `decay` in [0, 1]."""
    if not (np.isfinite(decay) and 0 <= decay <= 1):
        raise PMFMHDError("linear drag decay must be finite and in [0,1]")
    res = energy_compensation.data_ptr() if energy_compensation is not None else None
    _check(lib().pmfmhd_apply_linear_drag(context(s.device), ctypes.byref(s.grid), _p9(s.U), float(decay),
                                          _target(target_velocity), res, _stream()), "apply_linear_drag!")
    return s


def apply_exponential_drag_increment(s: MHDState, old_U, drag_impulse: float,
                                     target_velocity=(0.0, 0.0, 0.0)) -> MHDState:
    """drag.jl:121-208: exponential constant-force correction of the no-drag trial s.U."""
    _check_impulse(drag_impulse)
    if len(old_U) != NVAR:
        raise PMFMHDError(f"old_U must contain {NVAR} conserved fields")
    _check(lib().pmfmhd_apply_exponential_drag_increment(context(s.device), ctypes.byref(s.grid), _p9(s.U),
                                                         _p9(old_U), float(drag_impulse), _target(target_velocity),
                                                         _stream()), "apply_exponential_drag_increment!")
    return s


def step_drag_strang(s: MHDState, dt: float, drag_impulse: float, ch: Optional[float], glm_cr: float = 0.18,
                     integrator: str = "cube", target_velocity=(0.0, 0.0, 0.0)) -> MHDState:
    """drag.jl:218-228: exact half-step drag, one ideal-MHD step, exact half-step drag."""
    _check_impulse(drag_impulse)
    half_decay = float(np.exp(-0.5 * float(drag_impulse)))
    apply_linear_drag(s, half_decay, target_velocity)
    step(s, dt, ch=ch, glm_cr=glm_cr, integrator=integrator)
    apply_linear_drag(s, half_decay, target_velocity)
    return s


def step_drag_exponential(s: MHDState, dt: float, drag_impulse: float, ch: Optional[float], glm_cr: float = 0.18,
                          integrator: str = "cube", target_velocity=(0.0, 0.0, 0.0)) -> MHDState:
    """drag.jl:240-250: a no-drag trial step, then the exponential increment against the
    previous state (left in s.scratch by the ping-pong swap)."""
    _check_impulse(drag_impulse)
    step(s, dt, ch=ch, glm_cr=glm_cr, integrator=integrator)
    return apply_exponential_drag_increment(s, s.scratch, drag_impulse, target_velocity)


@dataclass
class DragRegimeController:
    """Hysteretic terminal / full-MHD regime switch (drag.jl:5-28)."""
    exit_drag_over_omega: float = 1.0
    enter_drag_over_omega: float = 2.0
    min_va_over_cs: float = 0.0
    confirm_checks: int = 2
    reenter_terminal: bool = False
    terminal: bool = False
    initialized: bool = False
    consecutive: int = 0

    def __post_init__(self):
        if not (0 < self.exit_drag_over_omega < self.enter_drag_over_omega):
            raise PMFMHDError("drag regime hysteresis requires 0 < exit < enter")
        if not self.min_va_over_cs >= 0:
            raise PMFMHDError("min_va_over_cs must be non-negative")
        if not self.confirm_checks >= 1:
            raise PMFMHDError("confirm_checks must be positive")
        self.exit_drag_over_omega = float(self.exit_drag_over_omega)
        self.enter_drag_over_omega = float(self.enter_drag_over_omega)
        self.min_va_over_cs = float(self.min_va_over_cs)
        self.confirm_checks = int(self.confirm_checks)


def update_drag_regime(controller: DragRegimeController, drag_over_omega: float, va_over_cs: float):
    """drag.jl:38-76: one sampled check; returns (terminal, transition) with transition in
    {"none", "terminal_to_full", "full_to_terminal"}. The handoff is one-way unless
    ``reenter_terminal``; every switch needs ``confirm_checks`` consecutive votes."""
    if not (np.isfinite(drag_over_omega) and drag_over_omega >= 0):
        raise PMFMHDError("drag_over_omega must be finite and non-negative")
    if not (np.isfinite(va_over_cs) and va_over_cs >= 0):
        raise PMFMHDError("va_over_cs must be finite and non-negative")
    c = controller
    ratio, mag = float(drag_over_omega), float(va_over_cs)
    if not c.initialized:
        c.terminal = mag >= c.min_va_over_cs and ratio >= c.enter_drag_over_omega
        c.initialized = True
        c.consecutive = 0
        return c.terminal, "none"
    if c.terminal:
        wants_full = mag < c.min_va_over_cs or ratio <= c.exit_drag_over_omega
        c.consecutive = c.consecutive + 1 if wants_full else 0
        if c.consecutive >= c.confirm_checks:
            c.terminal = False
            c.consecutive = 0
            return False, "terminal_to_full"
    elif c.reenter_terminal:
        wants_terminal = mag >= c.min_va_over_cs and ratio >= c.enter_drag_over_omega
        c.consecutive = c.consecutive + 1 if wants_terminal else 0
        if c.consecutive >= c.confirm_checks:
            c.terminal = True
            c.consecutive = 0
            return True, "full_to_terminal"
    else:
        c.consecutive = 0
    return c.terminal, "none"


def max_wavespeed(s: MHDState) -> float:
    out = ctypes.c_float()
    _check(lib().pmfmhd_max_wavespeed(context(s.device), ctypes.byref(s.grid), _p9(s.U), ctypes.byref(out),
                                      _stream()), "max_wavespeed")
    return out.value


def compute_dt(s: MHDState, cfl: float = 0.4):
    """(dt, smax) with dt = cfl*dx/max(smax, eps) (timestep.jl:37-46)."""
    dt, smax = ctypes.c_float(), ctypes.c_float()
    _check(lib().pmfmhd_compute_dt(context(s.device), ctypes.byref(s.grid), _p9(s.U), float(cfl), ctypes.byref(dt),
                                   ctypes.byref(smax), _stream()), "compute_dt")
    return dt.value, smax.value


def last_wavespeed(s: MHDState) -> float:
    out = ctypes.c_float()
    _check(lib().pmfmhd_last_wavespeed(context(s.device), ctypes.byref(out), _stream()), "last_wavespeed")
    return out.value


def evolve(s: MHDState, tfinal: float, cfl: float = 0.4, glm_ch_fac: float = 1.0, glm_cr: float = GLM_CR,
           integrator: Optional[str] = None, callback=None):
    """driver.jl:48-71: CFL-limited steps to ``tfinal``; returns (t, nsteps)."""
    if not glm_ch_fac > 0:
        raise PMFMHDError("glm_ch_fac must be positive")
    if not glm_cr >= 0:
        raise PMFMHDError("glm_cr must be non-negative")
    if integrator is None:
        integrator = "ref" if uses_ct(s) else "cube"
    T = np.float32
    t, n, tf = 0.0, 0, float(tfinal)
    while t < tf * (1 - 1e-9):
        dt, smax = compute_dt(s, cfl)
        if uses_ct(s):
            ch = T(0)
            dtf = float(dt)
        else:
            ch = T(T(glm_ch_fac) * T(smax))
            dtf = float(dt) * float(smax) / float(max(T(smax), ch))
        if t + dtf > tf:
            dtf = tf - t
        step(s, dtf, ch=float(ch), glm_cr=glm_cr, integrator=integrator)
        t += dtf
        n += 1
        if callback is not None:
            callback(s, t, n)
    return t, n


def run_glm(s: MHDState, nsteps: int, dt: float, ch: float, decay: float) -> MHDState:
    """nsteps fixed-dt GLM steps replayed from a cached CUDA graph; the state ends in s.U."""
    _check(lib().pmfmhd_run_glm(context(s.device), ctypes.byref(s.grid), _p9(s.U), _p9(s.scratch), int(nsteps),
                                float(dt), float(ch), float(decay), _resid_arg(s), _stream()), "run_glm")
    if nsteps % 2 == 1:
        s.U, s.scratch = s.scratch, s.U
    return s


def autotune(s: MHDState) -> None:
    _check(lib().pmfmhd_autotune(context(s.device), ctypes.byref(s.grid), _p9(s.U), 1 if uses_ct(s) else 0,
                                 1 if s.resid is not None else 0, _stream()), "autotune")


def set_tile(s: MHDState, rows: int, planes: int) -> None:
    """Pin the CTA tile (owned rows, z-planes per chunk) used for this state's grid."""
    _check(lib().pmfmhd_set_tile(context(s.device), ctypes.byref(s.grid), 1 if uses_ct(s) else 0,
                                 1 if s.resid is not None else 0, int(rows), int(planes)), "set_tile")


def get_tile(s: MHDState):
    rows, planes = ctypes.c_int(), ctypes.c_int()
    _check(lib().pmfmhd_get_tile(context(s.device), ctypes.byref(s.grid), 1 if uses_ct(s) else 0,
                                 1 if s.resid is not None else 0, ctypes.byref(rows), ctypes.byref(planes)),
           "get_tile")
    return rows.value, planes.value


def step_census(s: MHDState, dt: float, ch: float, decay: float) -> dict:
    """One GLM step (as step_cube; MC-PLM with HLLD, plain update) that also counts the HLLD
    single-star degeneracy cases over every face once: solves, sides with |denK| < 1e-12 (the
    reference's degenerate branch) and sides with 1e-12 <= |denK| < 1e-5 bn^2 (where the
    reference and relative tolerances give different fluxes)."""
    if uses_ct(s) or s.resid is not None:
        raise PMFMHDError("the census step is the plain GLM step")
    out = (ctypes.c_uint64 * 3)()
    _check(lib().pmfmhd_step_glm_census(context(s.device), ctypes.byref(s.grid), _p9(s.U), _p9(s.scratch),
                                        float(dt), float(ch), float(decay), out, _stream()), "step_census")
    s.U, s.scratch = s.scratch, s.U
    return {"solves": int(out[0]), "ref_sides": int(out[1]), "rel_sides": int(out[2])}


def set_tma_stall(device: Optional[int], polls: int) -> None:
    """Test hook of the bounded TMA wait (pmfmhd_set_tma_stall): with polls > 0 the following
    steps on this device's context arm each TMA plane without its copies and give up after
    `polls` polls; 0 restores normal staging."""
    _check(lib().pmfmhd_set_tma_stall(context(device), int(polls)), "set_tma_stall")


def device_status(s: MHDState, clear: bool = True) -> int:
    """0, or the PMFMHD_ETIMEOUT code if a step's bounded TMA wait gave up since the last check."""
    return lib().pmfmhd_status(context(s.device), int(clear), _stream())


def max_divb(s: MHDState) -> float:
    out = ctypes.c_double()
    _check(lib().pmfmhd_max_divb(context(s.device), ctypes.byref(s.grid), _p9(s.U), ctypes.byref(out), _stream()),
           "max_divb")
    return out.value


def max_divb_face(s: MHDState) -> float:
    if not uses_ct(s):
        raise PMFMHDError("max_divb_face needs a CT state (mhd_solver=:ct)")
    out = ctypes.c_double()
    _check(lib().pmfmhd_max_divb_face(context(s.device), ctypes.byref(s.grid), s.ct.packed.data_ptr(),
                                      ctypes.byref(out), _stream()), "max_divb_face")
    return out.value


def conserved_totals(s: MHDState) -> dict:
    out = (ctypes.c_double * 8)()
    _check(lib().pmfmhd_conserved_totals(context(s.device), ctypes.byref(s.grid), _p9(s.U), out, _stream()),
           "conserved_totals")
    keys = ("mass", "momx", "momy", "momz", "energy", "Bx", "By", "Bz")
    return dict(zip(keys, list(out)))


def ct_faces_from_potential(s: MHDState, Ax, Ay, Az) -> MHDState:
    """ct.jl:332-345: faces = discrete curl of an edge potential, cell B = face average."""
    if not uses_ct(s):
        raise PMFMHDError("ct_faces_from_potential! needs a CT state (mhd_solver=:ct)")
    dev = torch.device("cuda", s.device)
    A = []
    for a in (Ax, Ay, Az):
        a = torch.as_tensor(np.asarray(a, dtype=np.float32).reshape(-1) if not torch.is_tensor(a) else a)
        if a.numel() != s.nc:
            raise PMFMHDError(f"vector-potential array has {a.numel()} entries, expected {s.nc}")
        A.append(a.to(dev, torch.float32).contiguous())
    _check(lib().pmfmhd_ct_faces_from_potential(context(s.device), ctypes.byref(s.grid),
                                                _P3(*[a.data_ptr() for a in A]), _p9(s.U), s.ct.packed.data_ptr(),
                                                _stream()), "ct_faces_from_potential!")
    torch.cuda.current_stream().synchronize()
    return s


def ct_install_faces(s: MHDState, bxf, byf, bzf) -> MHDState:
    """ct.jl:228-236 `_ct_install_faces!`: faces set, remainders zeroed, cell B = face
    average, E keeps the thermal pressure, psi = 0 (on the device)."""
    if not uses_ct(s):
        raise PMFMHDError("_ct_install_faces! needs a CT state (mhd_solver=:ct)")
    dev = s.U[0].device
    for d, f in enumerate((bxf, byf, bzf)):
        t = torch.as_tensor(np.asarray(f, dtype=np.float32).ravel()) if not isinstance(f, torch.Tensor) else f
        if t.numel() != s.nc:
            raise PMFMHDError(f"face array has {t.numel()} entries, expected {s.nc}")
        s.ct.slot(d).copy_(t.to(dev, torch.float32).reshape(-1))
    _check(lib().pmfmhd_ct_install_faces(context(s.device), ctypes.byref(s.grid), _p9(s.U), s.ct.packed.data_ptr(),
                                         _stream()), "_ct_install_faces!")
    return s


def ct_faces_from_cells(s: MHDState) -> dict:
    """ct.jl:246-308: project the cell B onto the CT-admissible subspace (FP64 cuFFT on the
    device), install the faces, cell B = face average, E keeps the thermal pressure, psi = 0."""
    if not uses_ct(s):
        raise PMFMHDError("ct_faces_from_cells! needs a CT state (mhd_solver=:ct)")
    st = (ctypes.c_double * 3)()
    _check(lib().pmfmhd_ct_faces_from_cells(context(s.device), ctypes.byref(s.grid), _p9(s.U),
                                            s.ct.packed.data_ptr(), st, _stream()), "ct_faces_from_cells!")
    return {"cell_b_rel_l2_change": st[0], "magnetic_energy_ratio": st[1], "max_divb_face_dx_over_brms": st[2]}


# ---- terminal-regime induction (lib/MHDKernels/src/terminal_ct.jl) ---------------------------

def _cubic(s, what):
    if not all(d == s.dims[0] for d in s.dims):
        raise PMFMHDError(f"{what} requires a cubic grid")


def terminal_magnetic_force(s: MHDState, fx, fy, fz, B=None):
    """terminal_ct.jl:99-106: centred conservative Maxwell-stress force of B (default s.U[5..7])."""
    _cubic(s, "terminal magnetic force")
    B = B if B is not None else (s.U[5], s.U[6], s.U[7])
    _check(lib().pmfmhd_terminal_magnetic_force(context(s.device), ctypes.byref(s.grid), _P3(*[b.data_ptr() for b in B]),
                                                _P3(fx.data_ptr(), fy.data_ptr(), fz.data_ptr()), None, _stream()),
           "terminal_magnetic_force!")
    return fx, fy, fz


def terminal_magnetic_force_split(s: MHDState, px, py, pz, tx, ty, tz, B=None):
    """terminal_ct.jl:117-126: magnetic pressure -grad(B^2/2) and the tension remainder."""
    _cubic(s, "terminal magnetic force")
    B = B if B is not None else (s.U[5], s.U[6], s.U[7])
    _check(lib().pmfmhd_terminal_magnetic_force(context(s.device), ctypes.byref(s.grid), _P3(*[b.data_ptr() for b in B]),
                                                _P3(tx.data_ptr(), ty.data_ptr(), tz.data_ptr()),
                                                _P3(px.data_ptr(), py.data_ptr(), pz.data_ptr()), _stream()),
           "terminal_magnetic_force_split!")
    return px, py, pz, tx, ty, tz


def terminal_velocity_max(s: MHDState, gamma_drag: float, pressure_coeff: float, vcap: float = float("inf")) -> float:
    """terminal_ct.jl:226-238."""
    _cubic(s, "terminal CT")
    out = ctypes.c_double()
    _check(lib().pmfmhd_terminal_velocity_max(context(s.device), ctypes.byref(s.grid), _p9(s.U), float(gamma_drag),
                                              float(pressure_coeff), float(vcap), ctypes.byref(out), _stream()),
           "terminal_velocity_max!")
    return out.value


def terminal_ct_induction(s: MHDState, dt: float, gamma_drag: float, pressure_coeff: float, cfl: float = 0.4,
                          dissipation: float = 0.05, dissipation_order: int = 4, vcap: float = float("inf"),
                          max_subcycles: int = 256, compensate: bool = True):
    """terminal_ct.jl:502-575: returns (nsubcycles, vmax, eta)."""
    _cubic(s, "terminal CT")
    if not 0 < cfl <= 1:
        raise PMFMHDError("terminal CT cfl must be in (0,1]")
    if not 0 <= dissipation <= 1:
        raise PMFMHDError("terminal CT dissipation must be in [0,1]")
    if dissipation_order not in (2, 4):
        raise PMFMHDError("terminal CT dissipation_order must be 2 or 4")
    nsub, vmax, eta = ctypes.c_int(), ctypes.c_double(), ctypes.c_double()
    ct = s.ct.packed.data_ptr() if uses_ct(s) else None
    rc = lib().pmfmhd_terminal_ct_induction(context(s.device), ctypes.byref(s.grid), _p9(s.U), _p9(s.scratch), ct,
                                            float(dt), float(gamma_drag), float(pressure_coeff), float(cfl),
                                            float(dissipation), int(dissipation_order), float(vcap), int(max_subcycles),
                                            int(bool(compensate)), ctypes.byref(nsub), ctypes.byref(vmax),
                                            ctypes.byref(eta), _stream())
    if rc == -5:
        raise PMFMHDError(f"terminal CT needs more than {max_subcycles} subcycles (limit {max_subcycles})")
    _check(rc, "terminal_ct_induction!")
    return nsub.value, vmax.value, eta.value


def terminal_ct_euler_from_cell_emf(s: MHDState, dt: float) -> None:
    """terminal_ct.jl:476-486: faces += dt curl(edge average of ct.ec*), compensated."""
    if not uses_ct(s):
        raise PMFMHDError("terminal_ct_euler_from_cell_emf! needs a CT state")
    _check(lib().pmfmhd_terminal_ct_euler_from_cell_emf(context(s.device), ctypes.byref(s.grid), _p9(s.U),
                                                        s.ct.packed.data_ptr(), float(dt), _stream()),
           "terminal_ct_euler_from_cell_emf!")


# ---- primordial magnetic field initial conditions (lib/MHDKernels/src/pmf.jl) ----------------

_REALIZATION = {"physical_hash": 1, "physical_hash_zero_phase": 2}


def pmf_batchelor_field(dims, box=1.0, brms=1.0, seed=1, kcut=None, kmin=0.0, kmax=None, energy_index=4.0,
                        cutoff_order=2.0, mode_lock_n=None, high_mode_lock_n=None, preserve_low_kmax=None,
                        preserve_low_kcut=None, normalization_kind="auto", curl_symbol="centered",
                        curl_reference_n=None, fixed_mode_power=False, mode_realization="physical_hash",
                        realization_box=None, minimum_cells_per_wavelength=None, invariant_axis=0, device=None,
                        out=None):
    """pmf.jl:300-591 on the device: returns (Bx, By, Bz, stats), three float32 device arrays of
    nx*ny*nz values (x fastest). ``out`` may give the three arrays to fill. Only the
    physical-hash realizations are provided (the reference's ``:legacy`` draws use Julia's
    MersenneTwister)."""
    nx, ny, nz = (int(d) for d in dims)
    mode = str(mode_realization).lower()
    if mode == "legacy":
        raise PMFMHDError("mode_realization=:legacy (Julia MersenneTwister draws) is not provided; "
                          "use :physical_hash or :physical_hash_zero_phase")
    if mode not in _REALIZATION:
        raise PMFMHDError("mode_realization must be :legacy, :physical_hash, or :physical_hash_zero_phase")
    norm = {"auto": 0, "total": 1, "total_band": 1, "total_band_rms": 1, "reference": 2, "reference_band": 2,
            "low_band": 2, "reference_band_rms": 2}.get(str(normalization_kind).lower())
    if norm is None:
        raise PMFMHDError("normalization_kind must be :total_band_rms or :reference_band_rms")
    curl = {"centered": 0, "continuum": 1, "spectral": 1}.get(str(curl_symbol))
    if curl is None:
        raise PMFMHDError("curl_symbol must be :centered or :continuum")
    p = PmfParams(nx, ny, nz, _REALIZATION[mode], int(seed), float(box), float(brms),
                  float(realization_box) if realization_box is not None else 0.0,
                  float(kcut) if kcut is not None else 0.0, float(kmin), float(kmax) if kmax is not None else 0.0,
                  float(energy_index), float(cutoff_order), curl, int(curl_reference_n or 0), int(bool(fixed_mode_power)),
                  int(invariant_axis), float(preserve_low_kmax) if preserve_low_kmax is not None else 0.0,
                  float(preserve_low_kcut) if preserve_low_kcut is not None else 0.0, norm, int(mode_lock_n or 0),
                  int(high_mode_lock_n or 0), 0,
                  float(minimum_cells_per_wavelength) if minimum_cells_per_wavelength is not None else 0.0)
    dev = torch.device("cuda", torch.cuda.current_device() if device is None else device)
    B = out if out is not None else [torch.empty(nx * ny * nz, dtype=torch.float32, device=dev) for _ in range(3)]
    st = (ctypes.c_double * 6)()
    _check(lib().pmfmhd_pmf_batchelor_field(context(dev.index), ctypes.byref(p), _P3(*[b.data_ptr() for b in B]), st,
                                            _stream()), "pmf_batchelor_field")
    stats = {"brms": float(brms), "brms_measured": st[0], "total_brms_measured": st[0],
             "reference_band_brms_measured": st[1], "normalization_brms_measured": st[2],
             "normalization_kind": "reference_band_rms" if (norm == 2 or (norm == 0 and preserve_low_kmax))
             else "total_band_rms", "box": float(box), "kcut": st[3], "kmax": st[4], "seed": int(seed),
             "energy_index": float(energy_index), "mode_realization": mode,
             "realization_box": float(realization_box) if realization_box is not None else float(box),
             "preserve_high_source_scale": st[5]}
    return B[0], B[1], B[2], stats


def _install_pmf(s: MHDState, rho0, p0):
    _check(lib().pmfmhd_pmf_install(context(s.device), ctypes.byref(s.grid), _p9(s.U), float(rho0), float(p0),
                                    _stream()), "_install_pmf_field!")
    return ct_faces_from_cells(s) if uses_ct(s) else None


def init_pmf_batchelor(s: MHDState, brms=None, b0_pG=None, Bunit_pG=1.0, rho0=1.0, p0=1.0, box=None, **kw) -> dict:
    """pmf.jl:602-642: uniform gas (rho0, p0, at rest, psi = 0) around a Batchelor field
    generated in place into s.U[5..7]; CT states get faces from ct_faces_from_cells."""
    if brms is None:
        if b0_pG is None:
            raise PMFMHDError("provide either brms code units or b0_pG")
        brms = float(b0_pG) / float(Bunit_pG)
    box = s.dims[0] * s.dx if box is None else box
    *_, stats = pmf_batchelor_field(s.dims, box=box, brms=brms, device=s.device, out=[s.U[5], s.U[6], s.U[7]], **kw)
    ctinfo = _install_pmf(s, rho0, p0)
    stats.update(rho0=float(rho0), p0=float(p0), Bunit_pG=float(Bunit_pG))
    if ctinfo is not None:
        stats["ct_faces"] = ctinfo
    return stats


def init_pmf_batchelor_tiled(s: MHDState, tile_box, tile_n=None, brms=None, b0_pG=None, Bunit_pG=1.0, rho0=1.0,
                             p0=1.0, box=None, **kw) -> dict:
    """pmf.jl:652-700: a field generated on a smaller periodic tile of side tile_box (tile_n
    cells) and repeated through the box."""
    if brms is None:
        if b0_pG is None:
            raise PMFMHDError("provide either brms code units or b0_pG")
        brms = float(b0_pG) / float(Bunit_pG)
    L = float(s.dims[0] * s.dx if box is None else box)
    Lt = float(tile_box)
    if not Lt > 0:
        raise PMFMHDError("tile_box must be positive")
    if not Lt <= L:
        raise PMFMHDError("tile_box cannot exceed full box")
    n = s.dims[0]
    nt = int(round(n * Lt / L)) if tile_n is None else int(tile_n)
    if nt <= 0:
        raise PMFMHDError("tile_n must be positive")
    if nt > n:
        raise PMFMHDError("tile_n cannot exceed target grid size")
    if n % nt:
        raise PMFMHDError(f"tile_n={nt} must divide target grid size {n}")
    if not abs(Lt / L - nt / n) <= 4 * np.finfo(float).eps * max(1, Lt / L):
        raise PMFMHDError("tile_box/full box must match tile_n/target_n")
    Bt = pmf_batchelor_field((nt, nt, nt), box=Lt, brms=brms, device=s.device, **kw)
    nx, ny, nz = s.dims
    for d in range(3):
        _check(lib().pmfmhd_periodic_tile(context(s.device), Bt[d].data_ptr(), nt, nt, nt, s.U[5 + d].data_ptr(),
                                          nx, ny, nz, _stream()), "_periodic_tile_field")
    stats = dict(Bt[3])
    ctinfo = _install_pmf(s, rho0, p0)
    stats.update(rho0=float(rho0), p0=float(p0), Bunit_pG=float(Bunit_pG), full_box=L, tile_box=Lt, tile_n=nt)
    if ctinfo is not None:
        stats["ct_faces"] = ctinfo
    return stats


# ---- batched boxes ---------------------------------------------------------------------
class Batch:
    """Many independent periodic boxes advanced together (pmfmhd_batch_*)."""

    def __init__(self, states, cfl=0.2, glm_ch_fac=1.0, glm_cr=GLM_CR, device=None):
        self.states = list(states)
        boxes = (Box * len(self.states))()
        for b, s in zip(boxes, self.states):
            b.grid = s.grid
            b.U = _P9(*[t.data_ptr() for t in s.U])
            b.scratch = _P9(*[t.data_ptr() for t in s.scratch])
            b.ct_packed = s.ct.packed.data_ptr() if s.ct is not None else None
            b.resid = _P7(*([t.data_ptr() for t in s.resid] if s.resid is not None else [None] * 7))
            b.mhd_solver = 1 if s.ct is not None else 0
            b.cfl, b.glm_ch_fac, b.glm_cr = cfl, glm_ch_fac, glm_cr
        self._boxes = boxes
        self.device = self.states[0].device if device is None else device
        h = _VP()
        _check(lib().pmfmhd_batch_create(context(self.device), boxes, len(self.states), ctypes.byref(h)),
               "batch_create")
        self.handle = h

    def step(self, nsteps=1):
        _check(lib().pmfmhd_batch_step(self.handle, int(nsteps), _stream()), "batch_step")

    def query(self):
        n = len(self.states)
        t = (ctypes.c_double * n)()
        par = (ctypes.c_int32 * n)()
        dt = (ctypes.c_float * n)()
        _check(lib().pmfmhd_batch_query(self.handle, t, par, dt), "batch_query")
        return np.array(t), np.array(par), np.array(dt)

    def current_fields(self, i):
        """Host copy of box i's current state (U or scratch, by the parity from query)."""
        _, par, _ = self.query()
        s = self.states[i]
        src = s.scratch if par[i] else s.U
        return torch.stack(src).cpu().numpy()

    def close(self):
        if self.handle:
            lib().pmfmhd_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
