"""The NumPy restatement of terminal_ct.jl reproduces the reference's own known answers
(test/inherited/test_terminal_ct.jl:157-217, test_terminal_ct_equivalence.jl:1-150) before
it is trusted as the checker of the device kernels."""
import numpy as np
import pytest

import problems
import terminal_oracle as to

f32 = np.float32


def test_maxwell_stress_force_known_answer():
    """test_terminal_ct.jl:157-192: for B = (0, B0 sin 2 pi x, 0) the force is
    -pi B0^2 sin 4 pi x, all of it magnetic pressure."""
    N, B0 = 64, f32(0.2)
    i, _, _ = problems.cell_coords((N, N, N))
    by = (B0 * np.sin(np.pi * (f32(2) * ((i - 1) / N).astype(f32)))).astype(f32).reshape(N, N, N)
    B = [np.zeros_like(by), by, np.zeros_like(by)]
    inv2dx = f32(1) / (f32(2) * f32(1 / N))
    F = to.magnetic_force(B, inv2dx)
    P, Tn = to.magnetic_force_split(B, inv2dx)
    x = ((np.arange(N)) / N).astype(f32)
    exact = -f32(np.pi) * B0 ** 2 * np.sin(np.pi * (f32(4) * x))
    hfx = F[0][0, 0, :]
    assert np.sqrt(((hfx - exact) ** 2).sum() / (exact ** 2).sum()) < 0.01
    assert np.abs(F[1]).max() < 2e-6 and np.abs(F[2]).max() < 2e-6
    assert np.abs(P[0] - F[0]).max() < 2e-6
    assert max(np.abs(t).max() for t in Tn) < 2e-6
    rho, E, Bs = problems.terminal_seed(N)
    Bs = [b.reshape(N, N, N) for b in Bs]
    F = to.magnetic_force(Bs, inv2dx)
    P, Tn = to.magnetic_force_split(Bs, inv2dx)
    for d in range(3):
        assert np.all(np.abs((P[d] + Tn[d]) - F[d]) <= 2e-6 + 2e-6 * np.abs(F[d]))
    assert max(np.abs(t).max() for t in Tn) > 1e-5


def centred_div(B, dx):
    return ((to.sh(B[0], 0, 1) - to.sh(B[0], 0, -1)) + (to.sh(B[1], 1, 1) - to.sh(B[1], 1, -1)) +
            (to.sh(B[2], 2, 1) - to.sh(B[2], 2, -1))).astype(np.float64) / (2 * dx)


def test_induction_preserves_divergence_and_thermal_energy():
    """test_terminal_ct.jl:194-217: 8 terminal induction steps keep div B at round-off and
    the thermal energy unchanged."""
    N = 24
    rho, E, B = problems.terminal_seed(N)
    s = to.TerminalState(N, 1 / N, rho, E, B)
    eint0 = s.E - f32(0.5) * (s.B[0] ** 2 + s.B[1] ** 2 + s.B[2] ** 2)
    div0 = np.abs(centred_div(s.B, 1 / N)).max()
    b0 = s.B[0].copy()
    for _ in range(8):
        nsub, vmax, eta = s.induction(0.002, gamma_drag=4.0, pressure_coeff=0.2, cfl=0.4, dissipation=0.05,
                                      dissipation_order=4)
        assert nsub >= 1 and np.isfinite(vmax) and np.isfinite(eta)
    eint1 = s.E - f32(0.5) * (s.B[0] ** 2 + s.B[1] ** 2 + s.B[2] ** 2)
    div1 = np.abs(centred_div(s.B, 1 / N)).max()
    assert np.abs(s.B[0] - b0).max() > 1e-7
    assert div1 / N < 2e-6 and div1 <= max(8 * div0, 2e-5)
    assert np.abs(eint1 - eint0).max() < 2e-6


def run_pair(N, order, dtype, nsteps=20, dt=0.05):
    rho, B = problems.terminal_abc(N, dtype=dtype)
    T = np.dtype(dtype).type
    Bt = [b.astype(dtype) for b in B]
    E = T(1.5) + T(0.5) * (Bt[0] ** 2 + Bt[1] ** 2 + Bt[2] ** 2)
    glm = to.TerminalState(N, 1 / N, rho, E, Bt, dtype=dtype)
    # CT: faces = the (coordinate-independent) component values, cell B = face average = same
    ct = to.TerminalState(N, 1 / N, rho, E, Bt, faces=Bt, dtype=dtype)
    ct.B = to.face_average(ct.faces)
    kw = dict(gamma_drag=4.0, pressure_coeff=0.2, cfl=0.4, dissipation=0.05, dissipation_order=order)
    b0 = [b.astype(np.float64) for b in glm.B]
    for _ in range(nsteps):
        glm.induction(dt, **kw)
        ct.induction(dt, **kw)
    S = np.sqrt(sum(((glm.B[c] - b0[c]) ** 2).sum() for c in range(3)))
    d = np.sqrt(sum(((ct.B[c].astype(np.float64) - glm.B[c]) ** 2).sum() for c in range(3))) / S
    return d


@pytest.mark.parametrize("order", [4, 2])
def test_ct_and_glm_terminal_induction_converge_together(order):
    """test_terminal_ct_equivalence.jl:111-143 (FP64): the CT and GLM discretisations differ by
    O((k dx)^2): d(16) < 0.20, d(32) < 0.06, d(16)/d(32) > 3."""
    d16, d32 = run_pair(16, order, np.float64), run_pair(32, order, np.float64)
    assert d16 < 0.20 and d32 < 0.06 and d16 / d32 > 3
