"""Independent FP64 numpy restatement of the upstream CT prototype step used as a
cross-check in the reference's CT tests (test/inherited/test_ct.jl:7-144: MonCen
full slope, 3-direction Hancock predictor, HLL, Gardiner-Stone 2005 contact EMF, face
curl update) plus that test's analytic inputs (ct_test_potential :146-160,
ct_test_hydro :162-176). Test infrastructure: a second, structurally different
implementation (whole-array numpy, no per-cell loop) that pins the C++ oracle's CT path.

Arrays are indexed ``[k, j, i]`` (z, y, x) so that ``.ravel()`` gives the reference's
linidx order. Periodic neighbours are ``np.roll``.
"""
from __future__ import annotations

import numpy as np

SMALLR = 1e-6
SMALLP = 1e-6
AX = {0: -1, 1: -2, 2: -3}  # direction -> array axis (counted from the end)


def sh(a, d, s):
    """Value of the neighbour at offset ``s`` along direction ``d`` (periodic)."""
    return np.roll(a, -s, axis=AX[d])


def moncen(dl, dr):
    dc = 0.5 * (dl + dr)
    sg = np.where(dc >= 0.0, 1.0, -1.0)
    return np.where(dl * dr <= 0.0, 0.0, sg * np.minimum(2.0 * np.minimum(np.abs(dl), np.abs(dr)), np.abs(dc)))


def cellprim(U, bcc, g):
    rho = np.maximum(U[0], SMALLR)
    vx, vy, vz = U[1] / rho, U[2] / rho, U[3] / rho
    bx, by, bz = bcc
    p = np.maximum((g - 1) * (U[4] - 0.5 * rho * (vx * vx + vy * vy + vz * vz) - 0.5 * (bx * bx + by * by + bz * bz)), SMALLP)
    return np.stack([rho, vx, vy, vz, p, bx, by, bz])


def dflux(q, d, g):
    rho, vx, vy, vz, p, bx, by, bz = q
    b2 = bx * bx + by * by + bz * bz
    ptot = p + 0.5 * b2
    E = p / (g - 1) + 0.5 * rho * (vx * vx + vy * vy + vz * vz) + 0.5 * b2
    vb = vx * bx + vy * by + vz * bz
    v = (vx, vy, vz)
    b = (bx, by, bz)
    un, bn = v[d], b[d]
    out = [rho * un]
    for c in range(3):
        out.append(rho * un * v[c] - bn * b[c] + (ptot if c == d else 0.0))
    out.append((E + ptot) * un - bn * vb)
    for c in range(3):
        out.append(un * b[c] - (un * b[c] if c == d else v[c] * bn))
    return np.stack(out)


def fast_speed(q, d, g):
    rho = q[0]
    bn = q[5 + d]
    c2 = g * q[4] / rho
    b2 = (q[5] ** 2 + q[6] ** 2 + q[7] ** 2) / rho
    dd = 0.5 * (b2 + c2)
    return np.sqrt(dd + np.sqrt(np.maximum(dd * dd - c2 * bn * bn / rho, 0.0)))


def to_cons(q, g):
    rho, vx, vy, vz, p, bx, by, bz = q
    return np.stack([rho, rho * vx, rho * vy, rho * vz,
                     p / (g - 1) + 0.5 * rho * (vx * vx + vy * vy + vz * vz) + 0.5 * (bx * bx + by * by + bz * bz),
                     bx, by, bz])


def hll(L, R, d, g):
    cfL, cfR = fast_speed(L, d, g), fast_speed(R, d, g)
    uL, uR = L[1 + d], R[1 + d]
    SL = np.minimum(np.minimum(uL - cfL, uR - cfR), 0.0)
    SR = np.maximum(np.maximum(uL + cfL, uR + cfR), 0.0)
    FL, FR = dflux(L, d, g), dflux(R, d, g)
    UL, UR = to_cons(L, g), to_cons(R, g)
    return (SR * FL - SL * FR + SL * SR * (UR - UL)) / (SR - SL)


def hancock(U, bcc, dtdx, g):
    """Half-step primitive and per-direction full slopes of every cell."""
    q = cellprim(U, bcc, g)
    s = [moncen(q - sh(q, d, -1), sh(q, d, 1) - q) for d in range(3)]
    C = to_cons(q, g)
    acc = 0.0
    for d in range(3):
        acc = acc + (dflux(q + 0.5 * s[d], d, g) - dflux(q - 0.5 * s[d], d, g))
    Uh = C - 0.5 * dtdx * acc
    rho = np.maximum(Uh[0], SMALLR)
    vx, vy, vz = Uh[1] / rho, Uh[2] / rho, Uh[3] / rho
    bx, by, bz = Uh[5], Uh[6], Uh[7]
    p = np.maximum((g - 1) * (Uh[4] - 0.5 * rho * (vx * vx + vy * vy + vz * vz) - 0.5 * (bx * bx + by * by + bz * bz)), SMALLP)
    return np.stack([rho, vx, vy, vz, p, bx, by, bz]), s


def gs05(Ea0, Eam, Eb0, Ebm, mA0, mAm, mB0, mBm, Er00, Erm0, Er0m, Ermm):
    def up(m, lo, hi):
        return np.where(m > 0.0, lo, np.where(m < 0.0, hi, 0.5 * (lo + hi)))
    A1 = up(mA0, Erm0 - Ebm, Er00 - Eb0)
    A3 = up(mAm, Ebm - Ermm, Eb0 - Er0m)
    B1 = up(mB0, Er0m - Eam, Er00 - Ea0)
    B3 = up(mBm, Eam - Ermm, Ea0 - Erm0)
    return 0.25 * ((Ea0 + Eam + Eb0 + Ebm) + (A3 - A1) + (B3 - B1))


def fk_step(U, faces, dt, dx, g):
    """One CT step. ``U`` is (5, nz, ny, nx) (rho, m, E); ``faces`` is (3, nz, ny, nx). In place."""
    dtdx = dt / dx
    bcc = [0.5 * (faces[d] + sh(faces[d], d, 1)) for d in range(3)]
    Uc = np.concatenate([U, np.stack(bcc)])
    mh, s = hancock(Uc, bcc, dtdx, g)
    F = []
    for d in range(3):
        L = sh(mh + 0.5 * s[d], d, -1)
        R = mh - 0.5 * s[d]
        L = L.copy(); R = R.copy()
        L[0] = np.maximum(L[0], SMALLR); L[4] = np.maximum(L[4], SMALLP)
        R[0] = np.maximum(R[0], SMALLR); R[4] = np.maximum(R[4], SMALLP)
        L[5 + d] = faces[d]; R[5 + d] = faces[d]
        F.append(hll(L, R, d, g))
    Fx, Fy, Fz = F
    vx, vy, vz = mh[1], mh[2], mh[3]
    bx, by, bz = bcc
    e1, e2, e3 = vz * by - vy * bz, vx * bz - vz * bx, vy * bx - vx * by
    m = lambda a, d: sh(a, d, -1)  # value at the lower neighbour
    ez = gs05(-Fx[6], -m(Fx[6], 1), Fy[5], m(Fy[5], 0), Fx[0], m(Fx[0], 1), Fy[0], m(Fy[0], 0),
              e3, m(e3, 0), m(e3, 1), m(m(e3, 0), 1))
    ex = gs05(-Fy[7], -m(Fy[7], 2), Fz[6], m(Fz[6], 1), Fy[0], m(Fy[0], 2), Fz[0], m(Fz[0], 1),
              e1, m(e1, 1), m(e1, 2), m(m(e1, 1), 2))
    ey = gs05(-Fz[5], -m(Fz[5], 0), Fx[7], m(Fx[7], 2), Fz[0], m(Fz[0], 0), Fx[0], m(Fx[0], 2),
              e2, m(e2, 2), m(e2, 0), m(m(e2, 0), 2))
    for t in range(5):
        U[t] += dtdx * ((Fx[t] - sh(Fx[t], 0, 1)) + (Fy[t] - sh(Fy[t], 1, 1)) + (Fz[t] - sh(Fz[t], 2, 1)))
    faces[0] -= dtdx * ((sh(ez, 1, 1) - ez) - (sh(ey, 2, 1) - ey))
    faces[1] -= dtdx * ((sh(ex, 2, 1) - ex) - (sh(ez, 0, 1) - ez))
    faces[2] -= dtdx * ((sh(ey, 0, 1) - ey) - (sh(ex, 1, 1) - ex))


def ct_test_potential(N, amp=0.15):
    """Edge vector potential of a few Fourier modes (the reference test's input)."""
    dx = 1.0 / N
    tp = 2 * np.pi
    k, j, i = np.meshgrid(np.arange(1, N + 1), np.arange(1, N + 1), np.arange(1, N + 1), indexing="ij")
    xe, ye, ze = (i - 1) * dx, (j - 1) * dx, (k - 1) * dx
    Ax = amp * (np.sin(tp * ye + 0.3) * np.cos(tp * ze) + 0.5 * np.sin(tp * (ye + ze) + 1.0) / tp) / tp
    Ay = amp * (np.sin(tp * ze + 1.1) * np.cos(tp * xe + 0.4) + 0.4 * np.cos(tp * (xe - ze)) / tp) / tp
    Az = amp * (np.sin(tp * xe + 0.7) * np.cos(tp * ye + 0.2) + 0.3 * np.sin(tp * (xe + ye) + 0.5) / tp) / tp
    return np.stack([Ax.ravel(), Ay.ravel(), Az.ravel()])


def ct_test_hydro(N, g):
    """Conserved hydro part of the reference test's CT input (magnetic energy added later)."""
    tp = 2 * np.pi
    dx = 1.0 / N
    k, j, i = np.meshgrid(np.arange(1, N + 1), np.arange(1, N + 1), np.arange(1, N + 1), indexing="ij")
    x, y, z = (i - 0.5) * dx, (j - 0.5) * dx, (k - 0.5) * dx
    rho = 1 + 0.2 * np.sin(tp * x + 0.3) * np.cos(tp * y) + 0.1 * np.sin(tp * (y + z) + 0.9)
    vx = 0.3 * np.sin(tp * y + 0.1) + 0.1 * np.cos(tp * (x + z))
    vy = 0.3 * np.sin(tp * z + 0.8) + 0.1 * np.sin(tp * (x - y) + 0.2)
    vz = 0.3 * np.sin(tp * x + 0.5) + 0.1 * np.cos(tp * (y - z) + 0.6)
    p = 1 + 0.15 * np.cos(tp * (x + y) + 0.4) + 0.1 * np.sin(tp * z)
    U = np.zeros((9,) + rho.shape)
    U[0], U[1], U[2], U[3] = rho, rho * vx, rho * vy, rho * vz
    U[4] = p / (g - 1) + 0.5 * rho * (vx * vx + vy * vy + vz * vz)
    return U.reshape(9, -1)
