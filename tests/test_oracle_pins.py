"""The CPU oracle reproduces the reference's own logged known answers and its CT cross-check.

These pin the oracle (a C++ restatement of the reference scheme) before it is trusted as
the checker of the CUDA library. Known answers: docs/data/validation-cpu.log of the
reference (extracted to tests/golden/known_answers.json by tests/golden/make_known_answers.py).
"""
import numpy as np
import pytest

import fk_port
import oracle
import problems
from mhd_cases import KNOWN, alfven_L1


def _oracle_alfven(N, recon="plm", amp=0.1, p0=0.1, glm_cr=0.18):
    def make(dims, dx, recon_):
        s = oracle.OracleState(dims, dx, dtype=np.float32, recon=recon_)
        s.U[:] = problems.alfven_wave(dims, dx, amp=amp, B0=1.0, p0=p0)
        return s
    return alfven_L1(make, lambda s: s.U, lambda s: s.conserved_totals(),
                     lambda s, tf, cfl, cr: s.evolve(tf, cfl=cfl, glm_cr=cr), N, amp=amp, p0=p0, recon=recon,
                     glm_cr=glm_cr)


@pytest.mark.parametrize("recon", ["plm", "ppm"])
@pytest.mark.parametrize("N", [32, 64, 128])
def test_alfven_known_answer(recon, N):
    ref = KNOWN["alfven"][f"{recon}_{N}"]
    L1, n, t, drift = _oracle_alfven(N, recon)
    assert n == ref["steps"]
    assert abs(L1 / ref["L1"] - 1) < 0.02, (L1, ref["L1"])  # 2 significant digits of an f32 run
    assert drift["mass"] < 1e-4 and drift["energy"] < 1e-4


def test_alfven_convergence_order():
    L = [_oracle_alfven(N)[0] for N in (32, 64, 128)]
    orders = [np.log2(L[k - 1] / L[k]) for k in (1, 2)]
    assert all(o > 1.7 for o in orders), orders  # runtests.jl:48-55


def test_low_beta_alfven_known_answer():
    ref = KNOWN["alfven_lowbeta_64"]
    L1, n, _, drift = _oracle_alfven(64, p0=1e-3, glm_cr=1.0)
    assert n == ref["steps"]
    assert abs(L1 / ref["L1"] - 1) < 0.02
    assert drift["energy"] < 2e-4


def _brio_wu(N):
    s = oracle.OracleState((N, 4, 4), 1.0 / N, gamma=2.0, bcs=("outflow", "periodic", "periodic"))
    s.U[:] = problems.brio_wu((N, 4, 4), gamma=2.0)
    s.evolve(0.1, cfl=0.4)
    return s.U[0][:N].astype(np.float64)


def test_brio_wu_known_answer():
    ref = KNOWN["brio_wu"]
    r2, r4 = _brio_wu(256), _brio_wu(512)
    L1 = float(np.abs(r2 - 0.5 * (r4[0::2] + r4[1::2])).sum() / 256)
    assert abs(r2.min() - ref["rho_min"]) < 2e-3
    assert abs(L1 / ref["L1_256_vs_512"] - 1) < 0.02


def test_orszag_tang_known_answer():
    ref = KNOWN["orszag_tang_128"]
    N = 128
    s = oracle.OracleState((N, N, 1), 1.0 / N)
    s.U[:] = problems.orszag_tang((N, N, 1), 1.0 / N)
    t, n = s.evolve(0.5, cfl=0.4)
    h = s.U.astype(np.float64)
    brms = np.sqrt((h[5] ** 2 + h[6] ** 2 + h[7] ** 2).sum() / N ** 2)
    assert n == ref["steps"]
    assert abs(s.max_divb() * float(s.dx) / brms - ref["divb_dx_over_brms"]) < 0.1


def test_ct_matches_fork_port_fp64():
    """test/inherited/test_ct.jl:209-241 with an independent numpy restatement."""
    k = KNOWN["ct_fork_port"]
    N, g = k["N"], 5 / 3
    s = oracle.OracleState((N, N, N), 1 / N, dtype=np.float64, riemann="hll", recon="plm", mhd_solver="ct",
                           smallr=fk_port.SMALLR, pfl=fk_port.SMALLP)
    s.U[:] = fk_port.ct_test_hydro(N, g)
    s.ct_faces_from_potential(fk_port.ct_test_potential(N))
    assert s.max_divb_face() * float(s.dx) < 1e-13
    U = s.U[:5].reshape(5, N, N, N).copy()
    F = s.faces.reshape(3, N, N, N).copy()
    F0 = F.copy()
    dt, _ = s.compute_dt(k["cfl"])
    for _ in range(k["steps"]):
        s.step(dt)
        fk_port.fk_step(U, F, float(dt), 1 / N, g)
    rel = lambda a, b: np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)
    for t in range(5):
        assert rel(s.U[t].reshape(N, N, N), U[t]) < k["rel_tol"]
    for d in range(3):
        assert rel(s.faces[d].reshape(N, N, N), F[d]) < k["rel_tol"]
    assert rel(s.faces[0].reshape(N, N, N), F0[0]) > 1e-3
    assert s.max_divb_face() * float(s.dx) < 1e-12


def test_ct_divergence_preserved_fp32():
    """Face divergence stays at round-off through an evolution (test_ct.jl:336-375)."""
    N = 16
    s = oracle.OracleState((N, N, N), 1 / N, dtype=np.float32, mhd_solver="ct")
    s.U[:] = fk_port.ct_test_hydro(N, 5 / 3).astype(np.float32)
    s.ct_faces_from_potential(fk_port.ct_test_potential(N))
    brms = lambda: np.sqrt((s.U[5:8].astype(np.float64) ** 2).sum() / s.nc)
    divs = []
    s.evolve(0.1, cfl=0.3, callback=lambda st, t, n: divs.append(st.max_divb_face() * float(st.dx) / brms()))
    assert len(divs) > 5 and max(divs) < 1e-5
    assert np.all(s.U[8] == 0)


def test_oracle_f32_tracks_f64():
    """Same scheme in both precisions: smooth field, 10 steps, relative L-inf ~ f32 round-off."""
    n = 16
    U = problems.smooth_fields(n, dtype=np.float64)
    a = oracle.OracleState((n, n, n), 1 / n, dtype=np.float32)
    b = oracle.OracleState((n, n, n), 1 / n, dtype=np.float64)
    a.U[:] = U.astype(np.float32)
    b.U[:] = U
    dt, sp = b.compute_dt(0.2)
    for _ in range(10):
        a.step(dt, ch=sp)
        b.step(dt, ch=sp)
    for v in range(8):
        err = np.abs(a.U[v] - b.U[v]).max() / np.abs(b.U[v]).max()
        assert err < 2e-5, (v, err)


# ---- source-coupled drag (drag.jl, glm_physics.jl:63-172) ----------------------------------

@pytest.mark.parametrize("gamma_drag", [0.0, 100.0, 1000.0])
def test_drag_alfven_known_answer(gamma_drag):
    """test/inherited/test_drag_godunov.jl:16-57: a standing Alfven mode under linear drag
    follows the analytic damped oscillator (N=128x4x4, PPM/HLLD, dt=0.002 to t=0.1)."""
    N = 128
    s = oracle.OracleState((N, 4, 4), 1.0 / N, recon="ppm", riemann="hlld")
    s.U[:] = problems.drag_alfven(N)
    t = 0.0
    while t < 0.1 - 1e-14:
        dtn = min(0.002, 0.1 - t)
        s.step_drag_godunov(dtn, gamma_drag * dtn, ch=1.5, glm_cr=0.0)
        t += dtn
    i = np.arange(N)
    measured = 2.0 / N * np.sum(s.U[6][:N].astype(np.float64) * np.cos(2 * np.pi * (i + 0.5) / N))
    exact = 1e-3 * problems.drag_alfven_exact(t, gamma_drag, 2 * np.pi)
    assert np.isfinite(s.U[4]).all()
    assert abs(measured - exact) / 1e-3 < (0.015 if gamma_drag == 0 else 0.025)


@pytest.mark.parametrize("q", [1e-6, 1e-3, 0.1, 1.0, 10.0, 100.0])
def test_drag_uniform_state_work_known_answer(q):
    """test/inherited/test_terminal_ct.jl:343-370: on a uniform drifting state the step is
    pure drag: v -> v e^-q, the thermal energy is kept, the work is rho v^2 (1-e^-2q)/2 and
    the density is untouched."""
    n, rho, v, B, eth = 8, 1.5, (0.7, -0.2, 0.1), (0.3, -0.1, 0.2), 2.25
    s = oracle.OracleState((n, n, n), 1.0 / n, recon="ppm")
    s.U[:] = problems.uniform_drift(n, rho, v, B, eth)
    E0 = float(s.U[4][0])
    s.step_drag_godunov(0.01, q, ch=1.0, glm_cr=0.0)
    h = s.U.astype(np.float64)
    T = np.float32
    for d in range(3):
        assert abs(h[1 + d][0] / h[0][0] - v[d] * np.exp(-q)) <= 2e-7 + 5e-6 * abs(v[d] * np.exp(-q))
    ek = 0.5 * sum(h[1 + d][0] ** 2 for d in range(3)) / h[0][0]
    eb = 0.5 * sum(T(b) ** 2 for b in B)
    assert abs(h[4][0] - ek - eb - eth) <= 4e-6
    work = 0.5 * rho * sum(c * c for c in v) * (1 - np.exp(-2 * q))
    assert abs((E0 - h[4][0]) - work) <= 3e-7 + 8e-6 * work
    assert np.all(s.U[0] == T(rho))


def test_drag_zero_impulse_limit():
    """test/inherited/test_terminal_ct.jl:372-381: zero impulse reproduces the plain step."""
    n = 8
    U = problems.alfven_wave((n, n, n), 1.0 / n, amp=0.05, B0=1.0, p0=0.2)
    a = oracle.OracleState((n, n, n), 1.0 / n, recon="ppm")
    b = oracle.OracleState((n, n, n), 1.0 / n, recon="ppm")
    a.U[:] = U
    b.U[:] = U
    a.step(0.002, ch=1.5, glm_cr=0.3)
    b.step_drag_godunov(0.002, 0.0, ch=1.5, glm_cr=0.3)
    assert np.abs(a.U - b.U).max() < 2e-6


def test_drag_operators_limits():
    """apply_linear_drag with decay 1 and the exponential increment with impulse 0 leave a
    state unchanged up to the floors; decay 0 stops the gas in the target frame."""
    n = 6
    U = problems.turb_field((n, n, n), 1.0 / n)
    s = oracle.OracleState((n, n, n), 1.0 / n)
    s.U[:] = U
    s.apply_linear_drag(1.0)
    assert np.array_equal(s.U, U)
    s.apply_linear_drag(0.0, target_velocity=(0.1, 0.0, -0.2))
    assert np.allclose(s.U[1] / s.U[0], 0.1, atol=1e-7) and np.allclose(s.U[3] / s.U[0], -0.2, atol=1e-7)
    s.U[:] = U
    s.apply_exponential_drag_increment(U.copy(), 0.0)
    assert np.abs(s.U - U).max() <= 1e-6 * np.abs(U).max()
