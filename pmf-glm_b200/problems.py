"""Known-answer initial conditions for the MHD step (host-side numpy, not timed).

Each initialiser returns the nine conserved SoA fields ``U`` as a ``(9, nc)`` array
(rho, rho*vx, rho*vy, rho*vz, E, Bx, By, Bz, psi), cell ``(i, j, k)`` at
``((k*ny)+j)*nx+i`` with x fastest, matching the reference's ``linidx``.

Reference: lib/MHDKernels/src/problems.jl (turb field :9-29, Alfven :31-59,
Orszag-Tang :61-80, Brio-Wu :82-98, field loop :100-180) and the smooth parity field of
test/test_backends.jl:37-54.
"""
from __future__ import annotations

import numpy as np

NVAR = 9


def prim2cons(q, gamma):
    """glm_physics.jl:19-23 on stacked primitives ``q[9, ...]``."""
    rho, vx, vy, vz, p, bx, by, bz, psi = q
    E = p / (gamma - 1) + 0.5 * rho * (vx * vx + vy * vy + vz * vz) + 0.5 * (bx * bx + by * by + bz * bz)
    return np.stack([rho, rho * vx, rho * vy, rho * vz, E, bx, by, bz, psi])


def cell_coords(dims):
    """1-based (i, j, k) index grids flattened in linidx order (x fastest)."""
    nx, ny, nz = dims
    k, j, i = np.meshgrid(np.arange(1, nz + 1), np.arange(1, ny + 1), np.arange(1, nx + 1), indexing="ij")
    return i.ravel().astype(np.float64), j.ravel().astype(np.float64), k.ravel().astype(np.float64)


def _finish(q, gamma, dtype):
    return prim2cons(np.asarray(q, dtype=np.float64), gamma).astype(dtype)


def turb_field(dims, dx, gamma=5 / 3, dtype=np.float32):
    """Smooth field varying along all three axes (problems.jl:9-22)."""
    nx, ny, nz = dims
    i, j, k = cell_coords(dims)
    x = 2 * np.pi * (i - 0.5) / nx
    y = 2 * np.pi * (j - 0.5) / ny
    z = 2 * np.pi * (k - 0.5) / nz
    one = np.ones_like(x)
    q = [one, 0.2 * np.sin(z), 0.2 * np.sin(x), 0.2 * np.sin(y), one,
         0.3 + 0.1 * np.sin(2 * y), 0.1 * np.sin(2 * z), 0.1 * np.sin(2 * x), 0 * x]
    return _finish(q, gamma, dtype)


def alfven_wave(dims, dx, amp=1e-3, B0=1.0, p0=0.1, gamma=5 / 3, dtype=np.float32):
    """Right-going circularly polarised Alfven wave along x, vA = 1 (problems.jl:31-55)."""
    nx = dims[0]
    i, _, _ = cell_coords(dims)
    x = (i - 0.5) * dx
    L = nx * dx
    ph = 2 * np.pi / L * x
    by, bz = amp * np.sin(ph), amp * np.cos(ph)
    one = np.ones_like(x)
    q = [one, 0 * x, -by, -bz, p0 * one, B0 * one, by, bz, 0 * x]
    return _finish(q, gamma, dtype)


def alfven_by_exact(x, t, L, amp=1e-3):
    """problems.jl:57-59."""
    return amp * np.sin(2 * np.pi / L * np.mod(x - t, L))


def orszag_tang(dims, dx, gamma=5 / 3, dtype=np.float32):
    """2-D Orszag-Tang vortex (problems.jl:61-80)."""
    nx = dims[0]
    i, j, _ = cell_coords(dims)
    x = (i - 0.5) * dx
    y = (j - 0.5) * dx
    tp = 2 * np.pi / (nx * dx)
    one = np.ones_like(x)
    B0 = 1 / np.sqrt(4 * np.pi)
    q = [gamma * gamma * one, -np.sin(tp * y), np.sin(tp * x), 0 * x, gamma * one,
         -B0 * np.sin(tp * y), B0 * np.sin(2 * tp * x), 0 * x, 0 * x]
    return _finish(q, gamma, dtype)


def brio_wu(dims, gamma=2.0, dtype=np.float32):
    """Brio-Wu shock tube along x (problems.jl:82-98)."""
    nx = dims[0]
    i, _, _ = cell_coords(dims)
    left = i <= nx // 2
    one = np.ones_like(i)
    q = [np.where(left, 1.0, 0.125), 0 * i, 0 * i, 0 * i, np.where(left, 1.0, 0.1),
         0.75 * one, np.where(left, 1.0, -1.0), 0 * i, 0 * i]
    return _finish(q, gamma, dtype)


def field_loop(dims, dx, radius=0.3, amplitude=1e-3, rho0=1.0, p0=1.0, velocity=(1.0, 1.0, 0.0),
               gamma=5 / 3, dtype=np.float32):
    """Gardiner-Stone field-loop advection, GLM form (problems.jl:100-131).

    Returns ``(U, Az_edge)``; ``Az_edge`` is the edge-centred potential used to build CT faces.
    """
    nx, ny, nz = dims
    i, j, k = cell_coords(dims)
    # cell-centred A_z, then the centred discrete curl (problems.jl:100-131)
    x = (i - 0.5) * dx - 0.5 * nx * dx
    y = (j - 0.5) * dx - 0.5 * ny * dx
    A = (amplitude * np.maximum(radius - np.sqrt(x * x + y * y), 0.0)).astype(dtype).astype(np.float64)
    A3 = A.reshape(nz, ny, nx)
    bx = (np.roll(A3, -1, axis=1) - np.roll(A3, 1, axis=1)) / (2 * dx)
    by = -(np.roll(A3, -1, axis=2) - np.roll(A3, 1, axis=2)) / (2 * dx)
    one = np.ones_like(x)
    vx0, vy0, vz0 = velocity
    q = [rho0 * one, vx0 * one, vy0 * one, vz0 * one, p0 * one, bx.ravel(), by.ravel(), 0 * x, 0 * x]
    U = _finish(q, gamma, dtype)
    # edge-centred A_z at (i-1/2, j-1/2) (problems.jl:134-145)
    xe = (i - 1) * dx - 0.5 * nx * dx
    ye = (j - 1) * dx - 0.5 * ny * dx
    Az = amplitude * np.maximum(radius - np.sqrt(xe * xe + ye * ye), 0.0)
    return U, Az.astype(dtype)


def smooth_fields(n, gamma=5 / 3, dtype=np.float32):
    """Smooth parity field of the reference's backend tests (test_backends.jl:37-54)."""
    i, j, k = cell_coords((n, n, n))
    x = 2 * np.pi * (i - 0.5) / n
    y = 2 * np.pi * (j - 0.5) / n
    z = 2 * np.pi * (k - 0.5) / n
    q = [1 + 0.02 * np.sin(x) * np.cos(y), 0.02 * np.sin(z), 0.02 * np.sin(x), 0.02 * np.sin(y),
         1 + 0.01 * np.cos(z), 0.3 + 0.02 * np.sin(y), 0.02 * np.sin(z), 0.02 * np.sin(x), 0 * x]
    return _finish(q, gamma, dtype)
