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
