"""Terminal-regime induction on the device (terminal_ct.jl) through the C ABI: the
reference's known answers (test/inherited/test_terminal_ct.jl:157-217 and the CT/GLM
equivalence of test_terminal_ct_equivalence.jl) and parity with the NumPy oracle."""
import numpy as np
import pytest
import torch

import pmfmhd
import problems
import terminal_oracle as to

pytestmark = pytest.mark.gpu
f32 = np.float32
KW = dict(gamma_drag=4.0, pressure_coeff=0.2, cfl=0.4, dissipation=0.05)


def glm_state(N, rho, E, B):
    U = np.zeros((9, N ** 3), f32)
    U[0], U[4] = rho, E
    U[5:8] = np.stack(B)
    return pmfmhd.set_fields(pmfmhd.allocate_state((N, N, N), 1.0 / N), U)


def ct_state(N, rho, B):
    """CT state with faces = B (valid for fields whose components do not depend on their
    own coordinate), thermal energy 1.5, installed as _ct_install_faces! does."""
    U = np.zeros((9, N ** 3), f32)
    U[0], U[4] = rho, f32(1.5)
    s = pmfmhd.set_fields(pmfmhd.allocate_state((N, N, N), 1.0 / N, mhd_solver="ct"), U)
    return pmfmhd.ct_install_faces(s, B[0], B[1], B[2])


def test_maxwell_force_known_answer():
    """test_terminal_ct.jl:157-192."""
    N, B0 = 64, f32(0.2)
    i, _, _ = problems.cell_coords((N, N, N))
    by = (B0 * np.sin(np.pi * (f32(2) * ((i - 1) / N).astype(f32)))).astype(f32)
    z = np.zeros_like(by)
    s = glm_state(N, np.ones_like(by), np.ones_like(by), [z, by, z])
    F = [torch.empty(N ** 3, device="cuda") for _ in range(3)]
    P = [torch.empty(N ** 3, device="cuda") for _ in range(3)]
    Tn = [torch.empty(N ** 3, device="cuda") for _ in range(3)]
    pmfmhd.terminal_magnetic_force(s, *F)
    pmfmhd.terminal_magnetic_force_split(s, *P, *Tn)
    hf = [t.cpu().numpy() for t in F]
    x = (np.arange(N) / N).astype(f32)
    exact = -f32(np.pi) * B0 ** 2 * np.sin(np.pi * (f32(4) * x))
    assert np.sqrt(((hf[0][:N] - exact) ** 2).sum() / (exact ** 2).sum()) < 0.01
    assert np.abs(hf[1]).max() < 2e-6 and np.abs(hf[2]).max() < 2e-6
    assert np.abs(P[0].cpu().numpy() - hf[0]).max() < 2e-6
    assert max(t.abs().max().item() for t in Tn) < 2e-6
    rho, E, B = problems.terminal_seed(N)
    s = glm_state(N, rho, E, B)
    pmfmhd.terminal_magnetic_force(s, *F)
    pmfmhd.terminal_magnetic_force_split(s, *P, *Tn)
    for d in range(3):
        f, rec = F[d].cpu().numpy(), (P[d] + Tn[d]).cpu().numpy()
        assert np.all(np.abs(rec - f) <= 2e-6 + 2e-6 * np.abs(f))
    assert max(t.abs().max().item() for t in Tn) > 1e-5
    # against the oracle's force
    o = to.magnetic_force([b.reshape(N, N, N) for b in B], f32(1) / (f32(2) * f32(1 / N)))
    for d in range(3):
        assert np.abs(F[d].cpu().numpy() - o[d].ravel()).max() <= 1e-6 + 1e-5 * np.abs(o[d]).max()


def centred_div(h, N):
    B = [h[5 + d].astype(np.float64).reshape(N, N, N) for d in range(3)]
    return ((np.roll(B[0], -1, 2) - np.roll(B[0], 1, 2)) + (np.roll(B[1], -1, 1) - np.roll(B[1], 1, 1)) +
            (np.roll(B[2], -1, 0) - np.roll(B[2], 1, 0))) * (N / 2)


def test_induction_preserves_divergence_and_thermal_energy():
    """test_terminal_ct.jl:194-217, and parity with the oracle after the same 8 steps."""
    N = 24
    rho, E, B = problems.terminal_seed(N)
    s = glm_state(N, rho, E, B)
    o = to.TerminalState(N, 1 / N, rho, E, B)
    h0 = pmfmhd.fields_to_host(s)
    eint0 = h0[4] - f32(0.5) * (h0[5] ** 2 + h0[6] ** 2 + h0[7] ** 2)
    div0 = np.abs(centred_div(h0, N)).max()
    for _ in range(8):
        nsub, vmax, eta = pmfmhd.terminal_ct_induction(s, 0.002, dissipation_order=4, **KW)
        on, ov, oe = o.induction(0.002, dissipation_order=4, **KW)
        assert nsub == on and abs(vmax / ov - 1) < 1e-5 and abs(eta / oe - 1) < 1e-5
    h1 = pmfmhd.fields_to_host(s)
    eint1 = h1[4] - f32(0.5) * (h1[5] ** 2 + h1[6] ** 2 + h1[7] ** 2)
    div1 = np.abs(centred_div(h1, N)).max()
    assert np.abs(h1[5] - h0[5]).max() > 1e-7
    assert div1 / N < 2e-6 and div1 <= max(8 * div0, 2e-5)
    assert np.abs(eint1 - eint0).max() < 2e-6
    for d in range(3):
        ob = o.B[d].ravel()
        assert np.abs(h1[5 + d] - ob).max() <= 2e-7 + 5e-5 * np.abs(ob).max()
    assert np.array_equal(h1[0], h0[0])


def evolve(N, solver, order, nsteps=20, dt=0.05):
    rho, B = problems.terminal_abc(N, dtype=np.float32)
    if solver == "ct":
        s = ct_state(N, rho, B)
    else:
        s = glm_state(N, rho, f32(1.5) + f32(0.5) * (B[0] ** 2 + B[1] ** 2 + B[2] ** 2), B)
    h = pmfmhd.fields_to_host(s)
    b0 = h[5:8].astype(np.float64)
    et0 = h[4].astype(np.float64).sum()
    divmax = 0.0
    for _ in range(nsteps):
        pmfmhd.terminal_ct_induction(s, dt, dissipation_order=order, **KW)
        if solver == "ct":
            hb = pmfmhd.fields_to_host(s)[5:8].astype(np.float64)
            divmax = max(divmax, pmfmhd.max_divb_face(s) * s.dx / np.sqrt((hb ** 2).sum() / N ** 3))
    h = pmfmhd.fields_to_host(s)
    return b0, h[5:8].astype(np.float64), et0, h[4].astype(np.float64).sum(), divmax, s


@pytest.mark.parametrize("order", [4, 2])
def test_ct_and_glm_terminal_induction_equivalence(order):
    """test_terminal_ct_equivalence.jl:111-160 (Float32 form): CT and GLM differ by
    O((k dx)^2); CT keeps the face divergence at round-off and E follows the magnetic energy."""
    d = {}
    for N in (16, 32):
        g0, g1, _, _, _, _ = evolve(N, "glm", order)
        c0, c1, et0, et1, divmax, _ = evolve(N, "ct", order)
        S = np.sqrt(((g1 - g0) ** 2).sum())
        d[N] = np.sqrt(((c1 - g1) ** 2).sum()) / S
        dEm = 0.5 * ((c1 ** 2).sum() - (c0 ** 2).sum())
        assert divmax < 1e-5
        assert abs((et1 - et0) - dEm) / abs(et1) < 1e-5
    assert d[16] < 0.20 and d[32] < 0.06 and d[16] / d[32] > 3


def test_ct_terminal_matches_oracle_and_uses_remainders():
    N = 16
    rho, B = problems.terminal_abc(N, dtype=np.float32)
    s = ct_state(N, rho, B)
    h = pmfmhd.fields_to_host(s)
    o = to.TerminalState(N, 1 / N, rho, h[4], [h[5], h[6], h[7]], faces=B)
    for _ in range(3):
        pmfmhd.terminal_ct_induction(s, 0.05, dissipation_order=4, **KW)
        o.induction(0.05, dissipation_order=4, **KW)
    faces = s.ct.packed[: 3 * N ** 3].cpu().numpy().reshape(3, -1)
    for d in range(3):
        of = o.faces[d].ravel()
        assert np.abs(faces[d] - of).max() <= 2e-7 + 5e-5 * np.abs(of).max()
    h = pmfmhd.fields_to_host(s)
    assert np.abs(h[4] - o.E.ravel()).max() <= 2e-6 * np.abs(o.E).max()
    assert torch.count_nonzero(s.ct.rbx) > 0


def test_euler_from_cell_emf_matches_oracle():
    """terminal_ct.jl:461-486 with cell EMFs written into the CT workspace slots."""
    N = 16
    rho, B = problems.terminal_abc(N, dtype=np.float32)
    s = ct_state(N, rho, B)
    h = pmfmhd.fields_to_host(s)
    rng = np.random.default_rng(4)
    ec = (1e-3 * rng.standard_normal((3, N ** 3))).astype(f32)
    n = N ** 3
    for d in range(3):
        s.ct.slot(12 + d).copy_(torch.from_numpy(ec[d]).cuda())
    pmfmhd.terminal_ct_euler_from_cell_emf(s, 0.01)
    o = to.TerminalState(N, 1 / N, rho, h[4], [h[5], h[6], h[7]], faces=B)
    o.euler_from_cell_emf(ec, 0.01)
    faces = s.ct.packed[: 3 * n].cpu().numpy().reshape(3, -1)
    hb = pmfmhd.fields_to_host(s)
    for d in range(3):
        assert np.abs(faces[d] - o.faces[d].ravel()).max() <= 2e-7 + 1e-5 * np.abs(o.faces[d]).max()
        assert np.abs(hb[5 + d] - o.B[d].ravel()).max() <= 2e-7 + 1e-5 * np.abs(o.B[d]).max()
    assert np.abs(hb[4] - o.E.ravel()).max() <= 1e-6 * np.abs(o.E).max()
    assert np.all(hb[8] == 0)


def test_terminal_argument_errors():
    s = pmfmhd.allocate_state((16, 16, 8), 1.0 / 16)
    with pytest.raises(pmfmhd.PMFMHDError):
        pmfmhd.terminal_ct_induction(s, 0.01, **KW)
    c = glm_state(8, *problems.terminal_seed(8))
    with pytest.raises(pmfmhd.PMFMHDError):
        pmfmhd.terminal_ct_induction(c, 0.01, dissipation_order=3, **KW)
    with pytest.raises(pmfmhd.PMFMHDError):
        pmfmhd.terminal_ct_induction(c, 10.0, max_subcycles=1, dissipation_order=4, **KW)
