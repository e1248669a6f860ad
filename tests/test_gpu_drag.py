"""The source-coupled drag step and the split drag operators of the CUDA library (through
its C ABI) against the CPU oracle and the reference's own drag known answers:
test/test_backends.jl:76-121 (step_ref_drag! parity, q = 0.05), :353-374 (CT + drag),
test/inherited/test_drag_godunov.jl (drag-damped Alfven mode), test_terminal_ct.jl:343-385
(uniform-state work, zero limit, :cube with a moving target) and test_ct.jl:436-453 (CT
smoke, Strang / exponential wrappers with a moving target)."""
import numpy as np
import pytest
import torch

import oracle
import pmfmhd
import problems
from mhd_cases import KNOWN, within_parity

pytestmark = pytest.mark.gpu


def gpu_state(U, dims, dx=None, **kw):
    s = pmfmhd.allocate_state(dims, 1.0 / max(dims) if dx is None else dx, **kw)
    pmfmhd.set_fields(s, U)
    return s


def oracle_state(U, dims, dx=None, **kw):
    s = oracle.OracleState(dims, 1.0 / max(dims) if dx is None else dx, **kw)
    s.U[:] = U
    return s


@pytest.mark.parametrize("recon", ["plm", "ppm", "plm_minmod"])
@pytest.mark.parametrize("riemann", ["hlld", "hll", "llf"])
def test_glm_drag_matches_oracle(recon, riemann):
    """test_backends.jl:76-114: three step_ref_drag! steps, q = 0.05, N = 16 smooth field."""
    n = 16
    U = problems.smooth_fields(n)
    cpu = oracle_state(U, (n, n, n), recon=recon, riemann=riemann)
    dev = gpu_state(U, (n, n, n), recon=recon, riemann=riemann)
    dt, speed = cpu.compute_dt(0.08)
    for _ in range(3):
        cpu.step_drag_godunov(dt, 0.05, ch=speed)
        pmfmhd.step_drag_godunov(dev, float(dt), 0.05, ch=float(speed), integrator="ref")
    host = pmfmhd.fields_to_host(dev)
    assert not within_parity(cpu.U, host)
    assert host[0].min() > 0
    m0 = U[0].astype(np.float64).sum()
    assert abs(host[0].astype(np.float64).sum() / m0 - 1) < KNOWN["parity"]["mass_drift"]


@pytest.mark.parametrize("dims", [(37, 11, 5), (24, 24, 24)])
def test_glm_drag_moving_target_matches_oracle(dims):
    """A moving target frame and strong drag (q = 0.7) on a ragged and a cubic grid."""
    U = problems.turb_field(dims, 1.0 / max(dims))
    v0 = (0.05, -0.02, 0.01)
    cpu = oracle_state(U, dims)
    dev = gpu_state(U, dims)
    dt, speed = cpu.compute_dt(0.2)
    for _ in range(4):
        cpu.step_drag_godunov(dt, 0.7, ch=speed, target_velocity=v0)
        pmfmhd.step_drag_godunov(dev, float(dt), 0.7, ch=float(speed), integrator="ref", target_velocity=v0)
    assert not within_parity(cpu.U, pmfmhd.fields_to_host(dev))


@pytest.mark.parametrize("riemann", ["hlld", "hll"])
def test_ct_drag_matches_oracle(riemann):
    """test_backends.jl:353-374: CT steps then step_drag_godunov!(q = 0.2, :ref)."""
    n = 16
    dev = gpu_state(problems.smooth_fields(n), (n, n, n), riemann=riemann, mhd_solver="ct")
    pmfmhd.ct_faces_from_cells(dev)
    cpu = oracle_state(pmfmhd.fields_to_host(dev), (n, n, n), riemann=riemann, mhd_solver="ct")
    cpu.faces[:] = dev.ct.packed[: 3 * n ** 3].cpu().numpy().reshape(3, -1)
    m0 = cpu.U[0].astype(np.float64).sum()
    dt, _ = cpu.compute_dt(0.08)
    for _ in range(3):
        cpu.step(dt)
        pmfmhd.step(dev, float(dt), integrator="ref")
    cpu.step_drag_godunov(dt, 0.2, ch=0.0)
    pmfmhd.step_drag_godunov(dev, float(dt), 0.2, ch=0.0, integrator="ref")
    host = pmfmhd.fields_to_host(dev)
    assert not within_parity(cpu.U, host)
    faces = dev.ct.packed[: 3 * n ** 3].cpu().numpy().reshape(3, -1)
    for d in range(3):
        assert np.abs(faces[d] - cpu.faces[d]).max() <= 2e-6 + 5e-5 * np.abs(cpu.faces[d]).max()
    brms = np.sqrt((host[5:8].astype(np.float64) ** 2).sum() / n ** 3)
    assert pmfmhd.max_divb_face(dev) * dev.dx / brms < 1e-5
    assert abs(host[0].astype(np.float64).sum() / m0 - 1) < KNOWN["parity"]["mass_drift"]


@pytest.mark.parametrize("gamma_drag", [0.0, 100.0, 1000.0])
def test_drag_alfven_known_answer(gamma_drag):
    """test_drag_godunov.jl:16-57 on the GPU: the measured mode amplitude follows the
    analytic drag-damped oscillator, and matches the oracle's."""
    N = 128
    dev = gpu_state(problems.drag_alfven(N), (N, 4, 4), dx=1.0 / N, recon="ppm", riemann="hlld")
    cpu = oracle_state(problems.drag_alfven(N), (N, 4, 4), dx=1.0 / N, recon="ppm", riemann="hlld")
    t = 0.0
    while t < 0.1 - 1e-14:
        dtn = min(0.002, 0.1 - t)
        pmfmhd.step_drag_godunov(dev, dtn, gamma_drag * dtn, ch=1.5, glm_cr=0.0, integrator="ref")
        cpu.step_drag_godunov(dtn, gamma_drag * dtn, ch=1.5, glm_cr=0.0)
        t += dtn
    host = pmfmhd.fields_to_host(dev)
    i = np.arange(N)
    measured = 2.0 / N * np.sum(host[6][:N].astype(np.float64) * np.cos(2 * np.pi * (i + 0.5) / N))
    exact = 1e-3 * problems.drag_alfven_exact(t, gamma_drag, 2 * np.pi)
    assert np.isfinite(host[4]).all()
    assert abs(measured - exact) / 1e-3 < (0.015 if gamma_drag == 0 else 0.025)
    assert not within_parity(cpu.U, host)


@pytest.mark.parametrize("q", [1e-6, 1e-3, 0.1, 1.0, 10.0, 100.0])
def test_drag_uniform_state_work_known_answer(q):
    """test_terminal_ct.jl:343-370: v -> v e^-q, thermal energy kept, work
    rho v^2 (1 - e^-2q)/2 removed from E, density untouched."""
    n, rho, v, B, eth = 8, 1.5, (0.7, -0.2, 0.1), (0.3, -0.1, 0.2), 2.25
    dev = gpu_state(problems.uniform_drift(n, rho, v, B, eth), (n, n, n), recon="ppm")
    E0 = float(pmfmhd.fields_to_host(dev)[4][0])
    pmfmhd.step_drag_godunov(dev, 0.01, q, ch=1.0, glm_cr=0.0, integrator="ref")
    h32 = pmfmhd.fields_to_host(dev)
    h = h32.astype(np.float64)
    for d in range(3):
        assert abs(h[1 + d][0] / h[0][0] - v[d] * np.exp(-q)) <= 2e-7 + 5e-6 * abs(v[d] * np.exp(-q))
    ek = 0.5 * sum(h[1 + d][0] ** 2 for d in range(3)) / h[0][0]
    eb = 0.5 * sum(np.float32(b) ** 2 for b in B)
    assert abs(h[4][0] - ek - eb - eth) <= 4e-6
    work = 0.5 * rho * sum(c * c for c in v) * (1 - np.exp(-2 * q))
    assert abs((E0 - h[4][0]) - work) <= 3e-7 + 8e-6 * work
    assert np.all(h32[0] == np.float32(rho))
    assert np.isfinite(h32).all()


def test_drag_zero_impulse_limit_and_cube_errors():
    """test_terminal_ct.jl:372-385: q = 0 reproduces the plain step; the :cube drag step
    refuses a moving target and CT states; the impulse must be finite and >= 0."""
    n = 8
    U = problems.alfven_wave((n, n, n), 1.0 / n, amp=0.05, B0=1.0, p0=0.2)
    a = gpu_state(U, (n, n, n), recon="ppm")
    b = gpu_state(U, (n, n, n), recon="ppm")
    pmfmhd.step(a, 0.002, ch=1.5, glm_cr=0.3, integrator="ref")
    pmfmhd.step_drag_godunov(b, 0.002, 0.0, ch=1.5, glm_cr=0.3, integrator="ref")
    assert np.abs(pmfmhd.fields_to_host(a) - pmfmhd.fields_to_host(b)).max() < 2e-6
    with pytest.raises(pmfmhd.PMFMHDError):
        pmfmhd.step_drag_godunov(b, 0.002, 1.0, ch=1.5, integrator="cube", target_velocity=(0.1, 0, 0))
    for bad in (-1.0, float("nan"), float("inf")):
        with pytest.raises(pmfmhd.PMFMHDError):
            pmfmhd.step_drag_godunov(b, 0.002, bad, ch=1.5)
    with pytest.raises(pmfmhd.PMFMHDError):
        pmfmhd.step_drag_godunov(b, 0.002, 0.1, ch=1.5, integrator="rk2")
    with pytest.raises(pmfmhd.PMFMHDError):
        pmfmhd.apply_linear_drag(b, 1.5)
    c = gpu_state(problems.ct_smoke_fields(8), (8, 8, 8), riemann="hll", mhd_solver="ct")
    with pytest.raises(pmfmhd.PMFMHDError):
        pmfmhd.step_drag_godunov(c, 1e-3, 0.1, ch=1.0, integrator="cube")
    # the C ABI itself rejects a negative impulse (no launch)
    g = a.grid
    rc = pmfmhd.lib().pmfmhd_step_glm_drag(pmfmhd.context(a.device), pmfmhd.ctypes.byref(g), pmfmhd._p9(a.U),
                                           pmfmhd._p9(a.scratch), 0.002, 1.5, 1.0, -0.5, None, None)
    assert rc == -1


def test_ct_drag_smoke_and_split_wrappers():
    """test_ct.jl:436-453: four CT drag steps (q = 0.5) keep the face divergence at
    round-off; the Strang and exponential wrappers with a moving target stay finite and
    divergence-free."""
    N = 16
    s = gpu_state(problems.ct_smoke_fields(N), (N, N, N), riemann="hll", mhd_solver="ct")
    pmfmhd.ct_faces_from_cells(s)
    for _ in range(4):
        pmfmhd.step_drag_godunov(s, 2e-3, 0.5, ch=1.0, integrator="ref")
    h = pmfmhd.fields_to_host(s)
    d = pmfmhd.max_divb_face(s) * s.dx / np.sqrt((h[5].astype(np.float64) ** 2).mean())
    assert np.isfinite(h).all() and h[0].min() > 0
    assert d < 1e-5
    for f in (pmfmhd.step_drag_strang, pmfmhd.step_drag_exponential):
        s2 = gpu_state(problems.ct_smoke_fields(N), (N, N, N), riemann="hll", mhd_solver="ct")
        pmfmhd.ct_faces_from_cells(s2)
        f(s2, 2e-3, 0.4, ch=1.0, integrator="ref", target_velocity=(0.01, 0, 0))
        assert np.isfinite(pmfmhd.fields_to_host(s2)).all()
        assert pmfmhd.max_divb_face(s2) * s2.dx / 0.5 < 1e-5


@pytest.mark.parametrize("v0", [(0.0, 0.0, 0.0), (0.03, -0.01, 0.02)])
def test_split_drag_operators_match_oracle(v0):
    """apply_linear_drag (plain and energy-compensated) and the exponential increment
    against the oracle's elementwise restatement."""
    dims = (20, 12, 9)
    U = problems.turb_field(dims, 1.0 / 20)
    dev = gpu_state(U, dims)
    cpu = oracle_state(U, dims)
    pmfmhd.apply_linear_drag(dev, 0.8, v0)
    cpu.apply_linear_drag(0.8, v0)
    assert not within_parity(cpu.U, pmfmhd.fields_to_host(dev))
    res = torch.zeros(dev.nc, dtype=torch.float32, device=dev.U[0].device)
    res_h = np.zeros(dev.nc, np.float32)
    pmfmhd.apply_linear_drag(dev, 0.5, v0, energy_compensation=res)
    cpu.apply_linear_drag(0.5, v0, energy_residual=res_h)
    assert not within_parity(cpu.U, pmfmhd.fields_to_host(dev))
    assert np.abs(res.cpu().numpy() - res_h).max() <= 1e-6
    # exponential increment of a plain trial step against the state before it
    dt, speed = cpu.compute_dt(0.2)
    old_dev = [u.clone() for u in dev.U]
    old_cpu = cpu.U.copy()
    pmfmhd.step(dev, float(dt), ch=float(speed))
    cpu.step(dt, ch=speed)
    pmfmhd.apply_exponential_drag_increment(dev, old_dev, 2.0, v0)
    cpu.apply_exponential_drag_increment(old_cpu, 2.0, v0)
    assert not within_parity(cpu.U, pmfmhd.fields_to_host(dev))
