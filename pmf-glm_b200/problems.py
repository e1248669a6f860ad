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


def drag_alfven(N, amp=1e-3, gamma=5 / 3):
    """Standing Alfven mode of the drag test on an (N, 4, 4) grid, built in FP32 as the
    reference does (test/inherited/test_drag_godunov.jl:16-27): rho = 1, p0 = 1, B = (1, by, 0)
    with by = amp*cos(2 pi x), gas at rest."""
    T = np.float32
    dims = (N, 4, 4)
    i, _, _ = cell_coords(dims)
    x = ((i - 0.5) / N).astype(T)
    by = (T(amp) * np.cos(T(2 * np.pi) * x)).astype(T)
    U = np.zeros((9, x.size), T)
    U[0] = 1
    U[5] = 1
    U[6] = by
    U[4] = T(1) / (T(gamma) - T(1)) + T(0.5) * (T(1) + by * by)
    return U


def drag_alfven_exact(t, gamma_drag, kva):
    """Amplitude factor of a drag-damped standing Alfven mode (test_drag_godunov.jl:1-14)."""
    half = 0.5 * gamma_drag
    if gamma_drag == 0:
        return np.cos(kva * t)
    if half < kva:
        mu = np.sqrt(kva * kva - half * half)
        return np.exp(-half * t) * (np.cos(mu * t) + half / mu * np.sin(mu * t))
    if half > kva:
        mu = np.sqrt(half * half - kva * kva)
        rs, rf = -half + mu, -half - mu
        return (-rf * np.exp(rs * t) + rs * np.exp(rf * t)) / (rs - rf)
    return np.exp(-half * t) * (1 + half * t)


def uniform_drift(n, rho=1.5, v=(0.7, -0.2, 0.1), B=(0.3, -0.1, 0.2), etherm=2.25):
    """Uniform moving magnetised gas in FP32 (test/inherited/test_terminal_ct.jl:343-356)."""
    T = np.float32
    rho, etherm = T(rho), T(etherm)
    v = [T(c) for c in v]
    B = [T(c) for c in B]
    U = np.zeros((9, n ** 3), T)
    U[0] = rho
    for d in range(3):
        U[1 + d] = rho * v[d]
        U[5 + d] = B[d]
    U[4] = etherm + T(0.5) * rho * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) + T(0.5) * (
        B[0] * B[0] + B[1] * B[1] + B[2] * B[2])
    return U


def ct_smoke_fields(N, gamma=5 / 3):
    """Weakly perturbed CT smoke state (test/inherited/test_ct.jl:421-433), FP32."""
    T = np.float32
    g = T(gamma)
    i, j, _ = cell_coords((N, N, N))
    ph = (T(2) * T(np.pi) * (i - 1) / N).astype(T)
    ph2 = (T(2) * T(np.pi) * (j - 1) / N).astype(T)
    rho = T(1) + T(1e-2) * np.cos(ph)
    vx = T(1e-2) * np.sin(ph)
    bx = np.full_like(rho, T(0.5))
    by = T(0.05) * np.sin(ph)
    bz = T(0.03) * np.cos(ph2 + T(1))
    U = np.zeros((9, rho.size), T)
    U[0], U[1], U[5], U[6], U[7] = rho, rho * vx, bx, by, bz
    U[4] = T(1) / (g - T(1)) + T(0.5) * rho * vx * vx + T(0.5) * (bx * bx + by * by + bz * bz)
    return U


def ct_guide_problem(N, P0=1000.0, amp=2e-4, vamp=1e-4):
    """Weak oblique perturbation on a strong guide field (test/inherited/test_ct.jl:484-505):
    the edge potential (3, nc) and the hydro fields (5, nc: rho, momentum, E without magnetic
    energy), FP32 values of FP64 expressions accumulated in FP32 as the reference does. The
    faces are the staggered curl of the potential plus the guide field B0 = (35, 22, 28)."""
    T = np.float32
    i, j, k = cell_coords((N, N, N))
    x, y, z = (i - 1) / N, (j - 1) / N, (k - 1) / N
    modes = ((1, 2, -1, 0.3), (2, -1, 1, 1.1), (-1, 1, 2, 2.0), (3, 1, -2, 0.7), (1, -3, 2, 1.9))
    nc = N ** 3
    A = np.zeros((3, nc), T)
    rho = np.ones(nc, T)
    v = np.zeros((3, nc), T)
    amp, vamp = float(T(amp)), float(T(vamp))
    for m, (a, b, cc, ph) in enumerate(modes, start=1):
        arg = 2 * np.pi * (a * x + b * y + cc * z) + ph
        A[0] += (amp * np.sin(arg + m) / (2 * np.pi * (abs(b) + abs(cc)))).astype(T)
        A[1] += (amp * np.cos(arg) / (2 * np.pi * (abs(a) + abs(cc)))).astype(T)
        A[2] += (amp * np.sin(arg + 2 * m) / (2 * np.pi * (abs(a) + abs(b)))).astype(T)
        v[0] += (vamp * np.sin(arg + 0.5 * m)).astype(T)
        v[1] += (vamp * np.cos(arg + m)).astype(T)
        v[2] += (vamp * np.sin(arg + 1.5 * m)).astype(T)
        rho += (1e-3 * np.cos(arg + 2 * m)).astype(T)
    hyd = np.zeros((5, nc), T)
    hyd[0] = rho
    hyd[1:4] = rho * v
    hyd[4] = T(P0 / (5 / 3 - 1)) + T(0.5) * rho * (v[0] ** 2 + v[1] ** 2 + v[2] ** 2)
    return A, hyd, (T(35), T(22), T(28))


def terminal_seed(N, amp=0.08):
    """Terminal-regime seed state (test/inherited/test_terminal_ct.jl:133-155), FP32:
    rho = 1 + 0.02 sin(x+y), B = amp (sin y, sin z, sin x), thermal energy 1.5, gas at rest.
    Returns rho, E, (Bx, By, Bz) as flat arrays."""
    T = np.float32
    i, j, k = cell_coords((N, N, N))
    x = (2 * np.pi * (i - 1) / N).astype(T)
    y = (2 * np.pi * (j - 1) / N).astype(T)
    z = (2 * np.pi * (k - 1) / N).astype(T)
    rho = T(1) + T(0.02) * np.sin(x + y)
    B = [T(amp) * np.sin(y), T(amp) * np.sin(z), T(amp) * np.sin(x)]
    E = T(1.5) + T(0.5) * (B[0] ** 2 + B[1] ** 2 + B[2] ** 2)
    return rho.astype(T), E.astype(T), [b.astype(T) for b in B]


def terminal_abc(N, amp=0.08, dtype=np.float64):
    """ABC-type field of the CT/GLM terminal equivalence test
    (test/inherited/test_terminal_ct_equivalence.jl:40-62): each component independent of its
    own coordinate, so cell and face values coincide. Returns rho, (Bx, By, Bz) in `dtype`."""
    i, j, k = cell_coords((N, N, N))
    x, y, z = 2 * np.pi * (i - 1) / N, 2 * np.pi * (j - 1) / N, 2 * np.pi * (k - 1) / N
    rho = 1 + 0.02 * np.sin(x + y)
    B = [amp * (np.sin(y + 0.3) + 0.5 * np.cos(z)), amp * (np.sin(z + 0.7) + 0.5 * np.cos(x)),
         amp * (np.sin(x + 1.1) + 0.5 * np.cos(y))]
    return rho.astype(dtype), [b.astype(dtype) for b in B]
