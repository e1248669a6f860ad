"""ctypes wrapper of the CPU oracle (liboracle.so) — TEST INFRASTRUCTURE ONLY.

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use
this module, and only as the checker / the timed CPU baseline. The shipped library never
imports it.

``OracleState`` restates the reference's host driver: ``step!`` (driver.jl:20-37),
``evolve!`` (driver.jl:48-71), ``compute_dt`` (timestep.jl:37-46) and the diagnostics
(diagnostics.jl:6-55, ct.jl:176-201), with the scalar arithmetic done in the state's
precision T exactly where the reference does it in T.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

RECON = {"plm": 0, "ppm": 1, "plm_minmod": 2}
RIEMANN = {"hlld": 0, "hll": 1, "llf": 2}
BC = {"periodic": 0, "outflow": 1, "reflecting": 2}
GLM_CR = 0.18
N_WORK = 15
# HLLD single-star degeneracy test |denK| < max(1e-12, dtol_rel * bn^2): 0.0 is the reference's
# own test |denK| < 1e-12 (glm_physics.jl:257); 1e-5 is the relative test of the device
# library's default mode.
HLLD_DTOL_REFERENCE = 0.0
HLLD_DTOL_RELATIVE = 1e-5


class OracleParams(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("bc", ctypes.c_int * 3), ("recon", ctypes.c_int), ("riemann", ctypes.c_int),
                ("gamma", ctypes.c_double), ("smallr", ctypes.c_double), ("pfl", ctypes.c_double),
                ("llf_dmin", ctypes.c_double), ("llf_pmin", ctypes.c_double), ("hlld_dtol_rel", ctypes.c_double),
                ("zlo", ctypes.c_int), ("zhi", ctypes.c_int)]


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        _LIB = ctypes.CDLL(path)
        P = ctypes.POINTER(OracleParams)
        vp = ctypes.c_void_p
        d = ctypes.c_double
        for suf in ("f32", "f64"):
            getattr(_LIB, f"oracle_step_glm_{suf}").argtypes = [P, vp, vp, d, d, d, vp]
            getattr(_LIB, f"oracle_step_glm_census_{suf}").argtypes = [P, vp, vp, d, d, d, vp]
            getattr(_LIB, f"oracle_step_ct_{suf}").argtypes = [P, vp, vp, vp, vp, d, vp, vp]
            getattr(_LIB, f"oracle_step_glm_drag_{suf}").argtypes = [P, vp, vp, d, d, d, d, vp]
            getattr(_LIB, f"oracle_step_ct_drag_{suf}").argtypes = [P, vp, vp, vp, vp, d, d, vp]
            getattr(_LIB, f"oracle_step_glm_rad_{suf}").argtypes = [P, vp, vp, d, d, d, d, vp, ctypes.c_int]
            getattr(_LIB, f"oracle_step_ct_rad_{suf}").argtypes = [P, vp, vp, vp, vp, vp, d, d, vp, ctypes.c_int]
            for name in ("max_wavespeed",):
                f = getattr(_LIB, f"oracle_{name}_{suf}")
                f.argtypes = [P, vp]
                f.restype = d
            for name in ("max_divb", "max_divb_face"):
                f = getattr(_LIB, f"oracle_{name}_{suf}")
                f.argtypes = [P, vp, d]
                f.restype = d
            getattr(_LIB, f"oracle_ct_faces_from_potential_{suf}").argtypes = [P, vp, vp, vp, d]
            getattr(_LIB, f"oracle_totals_{suf}").argtypes = [P, vp, vp]
    return _LIB


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class OracleState:
    """Host mirror of the reference ``MHDState`` driven by the oracle."""

    def __init__(self, dims, dx, dtype=np.float32, gamma=5 / 3, smallr=1e-6, pfl=1e-7,
                 llf_dmin=1e-4, llf_pmin=0.0, riemann="hlld", recon="plm", bcs=("periodic",) * 3,
                 mhd_solver="glm", compensated=False, hlld_dtol_rel=HLLD_DTOL_RELATIVE):
        self.dims = tuple(int(d) for d in dims)
        self.nc = int(np.prod(self.dims))
        self.T = np.dtype(dtype).type
        self.dx = self.T(dx)
        self.gamma = self.T(gamma)
        self.mhd_solver = mhd_solver
        self.smallr = self.T(smallr)
        if mhd_solver == "ct" and any(b != "periodic" for b in bcs):
            raise ValueError("mhd_solver='ct' requires all-periodic boundaries")
        self.p = OracleParams(self.dims[0], self.dims[1], self.dims[2], (ctypes.c_int * 3)(*[BC[b] for b in bcs]),
                              RECON[recon], RIEMANN[riemann], float(self.gamma), float(self.T(smallr)),
                              float(self.T(pfl)), float(self.T(llf_dmin)), float(self.T(llf_pmin)),
                              float(self.T(hlld_dtol_rel)))
        self.U = np.zeros((9, self.nc), dtype=dtype)
        self.scratch = np.zeros_like(self.U)
        self.faces = np.zeros((3, self.nc), dtype=dtype) if mhd_solver == "ct" else None
        self.work = np.zeros((N_WORK, self.nc), dtype=dtype) if mhd_solver == "ct" else None
        self.resid = np.zeros((7, self.nc), dtype=dtype) if compensated else None
        self.face_resid = np.zeros((3, self.nc), dtype=dtype) if (compensated and mhd_solver == "ct") else None
        self._suf = "f32" if self.T is np.float32 else "f64"

    def _f(self, name):
        return getattr(lib(), f"oracle_{name}_{self._suf}")

    # -- the step (driver.jl:20-37, integrator_ref.jl:210-220, ct.jl:158-173) ----------------
    def step(self, dt, ch=None, glm_cr=GLM_CR):
        T = self.T
        dtdx = T(T(dt) / self.dx)
        if self.mhd_solver == "ct":
            self._f("step_ct")(ctypes.byref(self.p), _ptr(self.U), _ptr(self.scratch), _ptr(self.faces),
                               _ptr(self.work), float(dtdx), _ptr(self.resid), _ptr(self.face_resid))
        else:
            if ch is None:
                raise ValueError("step needs the GLM cleaning speed ch")
            decay = T(np.exp(T(-T(glm_cr) * T(ch) * T(dt) / self.dx)))
            self._f("step_glm")(ctypes.byref(self.p), _ptr(self.U), _ptr(self.scratch), float(dtdx),
                                float(T(ch)), float(decay), _ptr(self.resid))
        self.U, self.scratch = self.scratch, self.U

    def step_planes(self, dt, ch, zlo, zhi, glm_cr=GLM_CR):
        """The GLM step of planes [zlo, zhi) only, written into ``scratch`` without the swap: a
        bounded sample of a full step for timing the scheme on a large box."""
        T = self.T
        dtdx = T(T(dt) / self.dx)
        decay = T(np.exp(T(-T(glm_cr) * T(ch) * T(dt) / self.dx)))
        self.p.zlo, self.p.zhi = int(zlo), int(zhi)
        try:
            self._f("step_glm")(ctypes.byref(self.p), _ptr(self.U), _ptr(self.scratch), float(dtdx), float(T(ch)),
                                float(decay), _ptr(self.resid))
        finally:
            self.p.zlo, self.p.zhi = 0, 0

    def step_census(self, dt, ch, glm_cr=GLM_CR):
        """One GLM step (as ``step``) that also counts, over every face once, the HLLD solves,
        the single-star sides with |denK| < 1e-12 (the reference's degenerate branch) and those
        with 1e-12 <= |denK| < 1e-5 bn^2 (sent to the degenerate branch only by the relative
        test). Returns the three counts."""
        if self.mhd_solver != "glm":
            raise ValueError("the census step is the GLM step")
        T = self.T
        dtdx = T(T(dt) / self.dx)
        decay = T(np.exp(T(-T(glm_cr) * T(ch) * T(dt) / self.dx)))
        out = (ctypes.c_ulonglong * 3)()
        self._f("step_glm_census")(ctypes.byref(self.p), _ptr(self.U), _ptr(self.scratch), float(dtdx),
                                   float(T(ch)), float(decay), out)
        self.U, self.scratch = self.scratch, self.U
        return {"solves": int(out[0]), "ref_sides": int(out[1]), "rel_sides": int(out[2])}

    def step_drag_godunov(self, dt, drag_impulse, ch=None, glm_cr=GLM_CR, target_velocity=(0.0, 0.0, 0.0)):
        """Source-coupled Godunov step with linear drag (drag.jl:162-178, step_drag_godunov!;
        the kernel arithmetic of glm_physics.jl:63-172 and integrator_ref.jl:28-39,135,155-156
        is restated in mhd_oracle.cpp)."""
        if not (np.isfinite(drag_impulse) and drag_impulse >= 0):
            raise ValueError("drag impulse must be finite and non-negative")
        T = self.T
        dtdx = T(T(dt) / self.dx)
        v0 = (ctypes.c_double * 3)(*[float(T(v)) for v in target_velocity])
        if self.mhd_solver == "ct":
            self._f("step_ct_drag")(ctypes.byref(self.p), _ptr(self.U), _ptr(self.scratch), _ptr(self.faces),
                                    _ptr(self.work), float(dtdx), float(T(drag_impulse)), v0)
        else:
            decay = T(np.exp(T(-T(glm_cr) * T(ch) * T(dt) / self.dx)))
            self._f("step_glm_drag")(ctypes.byref(self.p), _ptr(self.U), _ptr(self.scratch), float(dtdx),
                                     float(T(ch)), float(decay), float(T(drag_impulse)), v0)
        self.U, self.scratch = self.scratch, self.U

    RAD_TRACK_DENSITY, RAD_TRACK_MAGNETIC, RAD_TRACK_ENERGY, RAD_CHECK, RAD_FIRST_ORDER = 1, 2, 4, 8, 16
    RAD_MASKED = 32

    def step_radiation(self, dt, drag_impulse, correction, ch=0.0, decay=1.0, track_density=True,
                       track_magnetic=True, track_energy=True, check_admissibility=False, robust_fallback=False,
                       global_fallback=False, fallback=False):
        """The radiation-coupled step kernel: step_ref_radiation! (integrator_ref.jl:238-258) and
        step_cube_radiation! (integrator_cube.jl:504-540). ``correction`` is the packed (9, nc)
        buffer of the state precision; its slot 0 is read as psi, slots 4-8 are updated.
        robust_fallback: minmod PLM with HLL; global_fallback: piecewise-constant states and LLF
        on every face, with the admissibility flag (CHECK == 3, integrator_cube.jl:168-177,
        524-529); fallback: the masked fallback (CHECK == 2, integrator_cube.jl:68-83,168-171):
        slot 4 as it is before the step is a per-cell mask, masked cells take zero offsets and
        faces touching them LLF, with the admissibility flag. The global fallback takes
        precedence (integrator_cube.jl:527)."""
        T = self.T
        corr = correction
        assert corr.dtype == self.U.dtype and corr.shape == (9, self.nc) and corr.flags["C_CONTIGUOUS"]
        masked = fallback and not global_fallback
        assert not (masked and self.mhd_solver == "ct"), "the masked fallback is a cube-kernel (GLM) mode"
        flags = ((self.RAD_TRACK_DENSITY if track_density else 0) | (self.RAD_TRACK_MAGNETIC if track_magnetic else 0)
                 | (self.RAD_TRACK_ENERGY if track_energy else 0)
                 | (self.RAD_CHECK if (check_admissibility or global_fallback or masked) else 0)
                 | (self.RAD_FIRST_ORDER if global_fallback else 0)
                 | (self.RAD_MASKED if masked else 0))
        saved = (self.p.recon, self.p.riemann)
        if robust_fallback:
            self.p.recon, self.p.riemann = RECON["plm_minmod"], RIEMANN["hll"]
        elif global_fallback:
            self.p.riemann = RIEMANN["llf"]
        Uin = np.concatenate([self.U[:8], corr[:1]])
        dtdx = T(T(dt) / self.dx)
        try:
            if self.mhd_solver == "ct":
                if self.face_resid is None:
                    self.face_resid = np.zeros((3, self.nc), dtype=self.U.dtype)
                self._f("step_ct_rad")(ctypes.byref(self.p), _ptr(Uin), _ptr(self.scratch), _ptr(self.faces),
                                       _ptr(self.work), _ptr(self.face_resid), float(dtdx), float(T(drag_impulse)),
                                       _ptr(corr), flags)
            else:
                self._f("step_glm_rad")(ctypes.byref(self.p), _ptr(Uin), _ptr(self.scratch), float(dtdx),
                                        float(T(ch)), float(T(decay)), float(T(drag_impulse)), _ptr(corr), flags)
        finally:
            self.p.recon, self.p.riemann = saved
        self.U, self.scratch = self.scratch, self.U

    def _drag_phi1(self, q):
        """glm_physics.jl:63-65 in the state precision."""
        T = self.T
        q = T(q)
        if abs(q) < T(1e-4):
            return T(T(T(1) - q / T(2)) + q * q / T(6))
        return T(-np.expm1(-q) / q)

    def apply_linear_drag(self, decay, target_velocity=(0.0, 0.0, 0.0), energy_residual=None):
        """apply_linear_drag! (drag.jl:78-117), elementwise in the state precision."""
        T = self.T
        with np.errstate(all="ignore"):
            U = self.U
            r = np.maximum(U[0], T(self.smallr))
            d = T(decay)
            ek0 = T(0.5) * (U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) / r
            for c in range(3):
                t = r * T(target_velocity[c])
                U[1 + c] = t + (U[1 + c] - t) * d
            ek1 = T(0.5) * (U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) / r
            if energy_residual is None:
                e = U[4] + (ek1 - ek0)
            else:
                inc = (ek1 - ek0) + energy_residual
                e = U[4] + inc
                energy_residual[:] = inc - (e - U[4])
            U[4] = np.maximum(e, T(1e-30))

    def apply_exponential_drag_increment(self, old_U, drag_impulse, target_velocity=(0.0, 0.0, 0.0)):
        """apply_exponential_drag_increment! (drag.jl:121-208) on the trial self.U."""
        T = self.T
        q = T(drag_impulse)
        decay, phi1 = T(np.exp(-q)), self._drag_phi1(q)
        with np.errstate(all="ignore"):
            U = self.U
            rn = np.maximum(U[0], T(self.smallr))
            ro = np.maximum(old_U[0], T(self.smallr))
            ek0 = T(0.5) * (U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) / rn
            eb = T(0.5) * (U[5] * U[5] + U[6] * U[6] + U[7] * U[7])
            nonkinetic = np.maximum(U[4] - ek0, eb + T(1e-30))
            for c in range(3):
                v0 = T(target_velocity[c])
                vo = old_U[1 + c] / ro
                vt = U[1 + c] / rn
                U[1 + c] = rn * (v0 + decay * (vo - v0) + phi1 * (vt - vo))
            ek1 = T(0.5) * (U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) / rn
            U[4] = np.maximum(nonkinetic + ek1, eb + T(1e-30))

    def max_wavespeed(self):
        return self.T(self._f("max_wavespeed")(ctypes.byref(self.p), _ptr(self.U)))

    def compute_dt(self, cfl=0.4):
        T = self.T
        smax = self.max_wavespeed()
        dt = T(T(cfl) * self.dx / max(smax, np.finfo(T).eps))
        return dt, smax

    def evolve(self, tfinal, cfl=0.4, glm_ch_fac=1.0, glm_cr=GLM_CR, callback=None):
        T = self.T
        t, n, tf = 0.0, 0, float(tfinal)
        while t < tf * (1 - 1e-9):
            dt, smax = self.compute_dt(cfl)
            if self.mhd_solver == "ct":
                ch = T(0)
                dtf = float(dt)
            else:
                ch = T(T(glm_ch_fac) * smax)
                dtf = float(dt) * float(smax) / float(max(smax, ch))
            if t + dtf > tf:
                dtf = tf - t
            self.step(dtf, ch=ch, glm_cr=glm_cr)
            t += dtf
            n += 1
            if callback is not None:
                callback(self, t, n)
        return t, n

    # -- diagnostics ----------------------------------------------------------------------
    def max_divb(self):
        return self._f("max_divb")(ctypes.byref(self.p), _ptr(self.U), float(self.dx))

    def max_divb_face(self):
        return self._f("max_divb_face")(ctypes.byref(self.p), _ptr(self.faces), float(self.dx))

    def conserved_totals(self):
        out = np.zeros(8)
        self._f("totals")(ctypes.byref(self.p), _ptr(self.U), _ptr(out))
        dV = float(self.dx * self.dx * self.dx)  # s.dx^3 in the state's precision (diagnostics.jl:45)
        keys = ("mass", "momx", "momy", "momz", "energy", "Bx", "By", "Bz")
        return {k: v * dV for k, v in zip(keys, out)}

    def ct_faces_from_potential(self, A):
        A = np.ascontiguousarray(np.asarray(A, dtype=self.U.dtype).reshape(3, self.nc))
        self._f("ct_faces_from_potential")(ctypes.byref(self.p), _ptr(A), _ptr(self.faces), _ptr(self.U),
                                           float(self.dx))
        if self.face_resid is not None:
            self.face_resid[:] = 0


def fallback_mask(trial_rho, dims, mask_in=None):
    """Fallback mask of the masked radiation step, in numpy: 1 where the trial density of the
    cell or of one of its six periodic face neighbours is negative (_radiation_fallback_mask_k!,
    radiation_coupling.jl:1536-1552), or, with ``mask_in``, where that mask is positive there
    as well (_radiation_expand_fallback_mask_k!, :1554-1577); 0 elsewhere. ``trial_rho`` and
    ``mask_in`` are flat in the SoA cell order (x fastest)."""
    nx, ny, nz = dims
    rho = np.asarray(trial_rho).reshape(nz, ny, nx)
    bad = rho < 0
    if mask_in is not None:
        bad = bad | (np.asarray(mask_in).reshape(nz, ny, nx) > 0)
    out = bad.copy()
    for axis in range(3):
        out |= np.roll(bad, 1, axis=axis) | np.roll(bad, -1, axis=axis)
    return out.astype(np.asarray(trial_rho).dtype).ravel()
