"""NumPy restatement of the terminal-regime induction (lib/MHDKernels/src/terminal_ct.jl) —
TEST INFRASTRUCTURE ONLY: the checker of the device kernels in libpmfmhd.so.

Fields are (N, N, N) arrays indexed [k, j, i] (x fastest, the reference's linidx order) in
the state precision; every operation is rounded in that precision in the reference's order
(its kernels use no @fastmath). ``np.roll(a, -1, axis)`` reads the +1 neighbour.
"""
from __future__ import annotations

import numpy as np

AX = {0: 2, 1: 1, 2: 0}  # x, y, z -> array axis


def sh(a, d, o):
    """a at (index + o) along direction d (periodic)."""
    return np.roll(a, -o, axis=AX[d])


def magnetic_force(B, inv2dx):
    """_tct_magnetic_force_at (terminal_ct.jl:18-51)."""
    T = B[0].dtype.type
    h = T(0.5)
    dt_ = [[None] * 3 for _ in range(3)]  # dt_[component][direction]
    for d in range(3):
        p = [sh(B[c], d, 1) for c in range(3)]
        m = [sh(B[c], d, -1) for c in range(3)]
        b2p = p[0] * p[0] + p[1] * p[1] + p[2] * p[2]
        b2m = m[0] * m[0] + m[1] * m[1] + m[2] * m[2]
        for c in range(3):
            if c == d:
                dt_[c][d] = (p[c] * p[c] - h * b2p) - (m[c] * m[c] - h * b2m)
            else:
                dt_[c][d] = p[c] * p[d] - m[c] * m[d]
    return [((dt_[c][0] + dt_[c][1]) + dt_[c][2]) * inv2dx for c in range(3)]


def magnetic_force_split(B, inv2dx):
    """_tct_magnetic_force_split_at (terminal_ct.jl:53-69): pressure and tension parts."""
    T = B[0].dtype.type
    F = magnetic_force(B, inv2dx)
    P = []
    for d in range(3):
        bp = [sh(B[c], d, 1) for c in range(3)]
        bm = [sh(B[c], d, -1) for c in range(3)]
        b2p = bp[0] * bp[0] + bp[1] * bp[1] + bp[2] * bp[2]
        b2m = bm[0] * bm[0] + bm[1] * bm[1] + bm[2] * bm[2]
        P.append(-T(0.5) * (b2p - b2m) * inv2dx)
    return P, [F[d] - P[d] for d in range(3)]


def velocity(rho, F, inv2dx, gamma_drag, pressure_coeff, smallr, vcap):
    """_tct_velocity_at (terminal_ct.jl:125-145)."""
    T = rho.dtype.type
    r = np.maximum(rho, T(smallr))
    g = [(T(pressure_coeff) * (sh(rho, d, 1) - sh(rho, d, -1))) * inv2dx for d in range(3)]
    gd = T(gamma_drag)
    invrg = T(1) / (r * max(gd, np.finfo(T).eps))
    v = [(F[d] - g[d]) * invrg for d in range(3)]
    v2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2]
    vc = T(vcap)
    with np.errstate(over="ignore", invalid="ignore", divide="ignore"):
        capped = v2 > vc * vc
        q = np.where(capped, vc / np.sqrt(v2), T(1)).astype(T)
    return [np.where(capped, v[d] * q, v[d]) for d in range(3)]


def emf(rho, F, B, inv2dx, gd, pc, smallr, vcap):
    """_tct_emf_at (terminal_ct.jl:147-155): e = v x B at every cell."""
    v = velocity(rho, F, inv2dx, gd, pc, smallr, vcap)
    return [v[1] * B[2] - v[2] * B[1], v[2] * B[0] - v[0] * B[2], v[0] * B[1] - v[1] * B[0]]


def lap(A, invdx2):
    T = A.dtype.type
    s = sh(A, 0, 1) + sh(A, 0, -1) + sh(A, 1, 1) + sh(A, 1, -1) + sh(A, 2, 1) + sh(A, 2, -1)
    return (s - T(6) * A) * invdx2


def bilap(A, invdx2):
    """_tct_bilap_at (terminal_ct.jl:166-181)."""
    T = A.dtype.type
    a1 = sh(A, 0, 1) + sh(A, 0, -1) + sh(A, 1, 1) + sh(A, 1, -1) + sh(A, 2, 1) + sh(A, 2, -1)
    a2 = sh(A, 0, 2) + sh(A, 0, -2) + sh(A, 1, 2) + sh(A, 1, -2) + sh(A, 2, 2) + sh(A, 2, -2)

    def d2(a, b, oa, ob):
        return sh(sh(A, a, oa), b, ob)
    diag = (d2(0, 1, 1, 1) + d2(0, 1, 1, -1) + d2(0, 1, -1, 1) + d2(0, 1, -1, -1) + d2(0, 2, 1, 1) +
            d2(0, 2, 1, -1) + d2(0, 2, -1, 1) + d2(0, 2, -1, -1) + d2(1, 2, 1, 1) + d2(1, 2, 1, -1) +
            d2(1, 2, -1, 1) + d2(1, 2, -1, -1))
    return ((T(42) * A - T(12) * a1) + a2 + T(2) * diag) * invdx2 * invdx2


def rhs_glm(e, B, inv2dx, invdx2, eta, order):
    """_tct_rhs_at (terminal_ct.jl:183-209): centred curl of the cell EMF plus dissipation."""
    dx = ((sh(e[2], 1, 1) - sh(e[2], 1, -1)) - (sh(e[1], 2, 1) - sh(e[1], 2, -1))) * inv2dx
    dy = ((sh(e[0], 2, 1) - sh(e[0], 2, -1)) - (sh(e[2], 0, 1) - sh(e[2], 0, -1))) * inv2dx
    dz = ((sh(e[1], 0, 1) - sh(e[1], 0, -1)) - (sh(e[0], 1, 1) - sh(e[0], 1, -1))) * inv2dx
    return [x - eta * bilap(B[c], invdx2) if order == 4 else x + eta * lap(B[c], invdx2)
            for c, x in enumerate((dx, dy, dz))]


def edges(ec):
    """_tctc_edge_k! (terminal_ct.jl:325-345): edge EMF = mean of the four cells at the edge."""
    T = ec[0].dtype.type
    q = T(0.25)
    ez = q * (((ec[2] + sh(ec[2], 0, -1)) + sh(ec[2], 1, -1)) + sh(sh(ec[2], 0, -1), 1, -1))
    ex = q * (((ec[0] + sh(ec[0], 1, -1)) + sh(ec[0], 2, -1)) + sh(sh(ec[0], 1, -1), 2, -1))
    ey = q * (((ec[1] + sh(ec[1], 0, -1)) + sh(ec[1], 2, -1)) + sh(sh(ec[1], 0, -1), 2, -1))
    return [ex, ey, ez]


def rate_faces(E, A, invdx, invdx2, eta, order):
    """_tctc_rate_at (terminal_ct.jl:347-362)."""
    ex, ey, ez = E
    dx = ((sh(ez, 1, 1) - ez) - (sh(ey, 2, 1) - ey)) * invdx
    dy = ((sh(ex, 2, 1) - ex) - (sh(ez, 0, 1) - ez)) * invdx
    dz = ((sh(ey, 0, 1) - ey) - (sh(ex, 1, 1) - ex)) * invdx
    return [x - eta * bilap(A[c], invdx2) if order == 4 else x + eta * lap(A[c], invdx2)
            for c, x in enumerate((dx, dy, dz))]


def face_average(f):
    T = f[0].dtype.type
    h = T(0.5)
    return [h * (f[0] + sh(f[0], 0, 1)), h * (f[1] + sh(f[1], 1, 1)), h * (f[2] + sh(f[2], 2, 1))]


def comp_update(x, dx, r):
    inc = dx + r
    upd = x + inc
    r[...] = inc - (upd - x)
    return upd


class TerminalState:
    """rho, E, cell B (and CT faces with their remainders) of a cubic periodic box."""

    def __init__(self, N, dx, rho, E, B, faces=None, dtype=np.float32, smallr=1e-6):
        T = np.dtype(dtype).type
        self.T, self.N, self.dx = T, N, T(dx)
        sh3 = (N, N, N)
        self.rho = np.asarray(rho, T).reshape(sh3).copy()
        self.E = np.asarray(E, T).reshape(sh3).copy()
        self.B = [np.asarray(b, T).reshape(sh3).copy() for b in B]
        self.faces = None if faces is None else [np.asarray(f, T).reshape(sh3).copy() for f in faces]
        self.rb = None if faces is None else [np.zeros(sh3, T) for _ in range(3)]
        self.smallr = T(smallr)

    def velocity_max(self, gamma_drag, pressure_coeff, vcap=np.inf):
        """terminal_velocity_max! (terminal_ct.jl:226-238)."""
        T = self.T
        inv2dx = T(1) / (T(2) * self.dx)
        F = magnetic_force(self.B, inv2dx)
        v = velocity(self.rho, F, inv2dx, gamma_drag, pressure_coeff, self.smallr, vcap)
        return float(np.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]).max())

    def induction(self, dt, gamma_drag, pressure_coeff, cfl=0.4, dissipation=0.05, dissipation_order=4,
                  vcap=np.inf, max_subcycles=256, compensate=True):
        """terminal_ct_induction! (terminal_ct.jl:502-551, subcycles :553-575)."""
        T, dx = self.T, self.dx
        inv2dx = T(1) / (T(2) * dx)
        invdx = T(1) / dx
        invdx2 = T(1) / (dx * dx)
        vmax = self.velocity_max(gamma_drag, pressure_coeff, vcap)
        nsub = max(1, int(np.ceil(float(dt) * vmax / max(float(cfl) * float(dx), np.finfo(float).eps))))
        if nsub > max_subcycles:
            raise ValueError(f"terminal CT needs {nsub} subcycles (limit {max_subcycles})")
        dts = T(dt / nsub)
        order = dissipation_order
        eta = (T(dissipation / 12) * T(vmax) * (dx * dx * dx) if order == 4 else T(dissipation) * T(vmax) * dx)
        args = (inv2dx, gamma_drag, pressure_coeff, self.smallr, vcap)
        small = T(1e-30)
        h = T(0.5)
        for _ in range(nsub):
            if self.faces is None:
                e = emf(self.rho, magnetic_force(self.B, inv2dx), self.B, *args)
                r = rhs_glm(e, self.B, inv2dx, invdx2, eta, order)
                pB = [self.B[c] + dts * r[c] for c in range(3)]
                e = emf(self.rho, magnetic_force(pB, inv2dx), pB, *args)
                r = rhs_glm(e, pB, inv2dx, invdx2, eta, order)
                nB = [h * ((self.B[c] + pB[c]) + dts * r[c]) for c in range(3)]
            else:
                e = emf(self.rho, magnetic_force(self.B, inv2dx), self.B, *args)
                r = rate_faces(edges(e), self.faces, invdx, invdx2, eta, order)
                pf = [self.faces[c] + dts * r[c] for c in range(3)]
                pB = face_average(pf)
                e = emf(self.rho, magnetic_force(pB, inv2dx), pB, *args)
                r = rate_faces(edges(e), pf, invdx, invdx2, eta, order)
                for c in range(3):
                    ob = self.faces[c]
                    if compensate:
                        self.faces[c] = comp_update(ob, h * ((pf[c] - ob) + dts * r[c]), self.rb[c])
                    else:
                        self.faces[c] = h * ((ob + pf[c]) + dts * r[c])
                nB = face_average(self.faces)
            ob = self.B
            eb0 = h * (ob[0] * ob[0] + ob[1] * ob[1] + ob[2] * ob[2])
            eb1 = h * (nB[0] * nB[0] + nB[1] * nB[1] + nB[2] * nB[2])
            self.B = nB
            self.E = np.maximum((self.E + eb1) - eb0, small)
        return nsub, vmax, float(eta)

    def euler_from_cell_emf(self, ec, dt):
        """terminal_ct_euler_from_cell_emf! (terminal_ct.jl:461-486): edges of the given cell
        EMFs, compensated face update, cell B = face average with E following."""
        T = self.T
        E = edges([np.asarray(x, T).reshape(self.N, self.N, self.N) for x in ec])
        invdx = T(1) / self.dx
        dtt = T(dt)
        ex, ey, ez = E
        rates = [((sh(ez, 1, 1) - ez) - (sh(ey, 2, 1) - ey)), ((sh(ex, 2, 1) - ex) - (sh(ez, 0, 1) - ez)),
                 ((sh(ey, 0, 1) - ey) - (sh(ex, 1, 1) - ex))]
        for c in range(3):
            self.faces[c] = comp_update(self.faces[c], dtt * rates[c] * invdx, self.rb[c])
        nB = face_average(self.faces)
        h = T(0.5)
        ob = self.B
        self.E = self.E + h * ((nB[0] * nB[0] + nB[1] * nB[1] + nB[2] * nB[2]) - (ob[0] * ob[0] + ob[1] * ob[1] + ob[2] * ob[2]))
        self.B = nB
