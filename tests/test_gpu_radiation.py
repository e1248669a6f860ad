"""The radiation-coupled step of the CUDA library (pmfmhd_step_radiation: the drag step
with per-cell velocity corrections, tracked density increments, Kahan remainders of E and
B, the admissibility flag and the fallback schemes) against the CPU oracle, and the
reference's guide-field known answer for compensated CT faces
(test/inherited/test_ct.jl:476-567), which runs this kernel with and without
track_magnetic. Parity gates follow test/test_backends.jl:65-121."""
import numpy as np
import pytest
import torch

import oracle
import pmfmhd
import problems
from mhd_cases import within_parity

pytestmark = pytest.mark.gpu
f32 = np.float32


def gpu_state(U, dims, **kw):
    s = pmfmhd.allocate_state(dims, 1.0 / max(dims), **kw)
    pmfmhd.set_fields(s, U)
    return s


def corrections(nc, seed, psi, scale=2e-3):
    """A packed correction buffer: psi in slot 0, smooth-ish random velocity corrections in
    slots 1-3, small nonzero remainders/perturbation in 4-8 (so that tracking reads them)."""
    rng = np.random.default_rng(seed)
    c = np.zeros((9, nc), f32)
    c[0] = psi
    c[1:4] = (scale * rng.standard_normal((3, nc))).astype(f32)
    c[4] = (1e-3 * rng.standard_normal(nc)).astype(f32)
    c[5:9] = (1e-8 * rng.standard_normal((4, nc))).astype(f32)
    return c


def corr_parity(a, b):
    for v in range(9):
        assert np.abs(a[v] - b[v]).max() <= 2e-6 + 5e-5 * np.abs(b[v]).max(), v


@pytest.mark.parametrize("flags", [dict(track_density=True, track_magnetic=True, track_energy=True),
                                   dict(track_density=False, track_magnetic=False, track_energy=False),
                                   dict(track_density=True, track_magnetic=False, track_energy=True)])
@pytest.mark.parametrize("recon,riemann", [("plm", "hlld"), ("ppm", "hll"), ("plm", "llf")])
def test_glm_radiation_matches_oracle(flags, recon, riemann):
    n = 16
    U = problems.smooth_fields(n)
    U[8] = (1e-3 * np.sin(np.arange(n ** 3) * 0.37)).astype(f32)  # nonzero psi in slot 0
    cpu = oracle.OracleState((n, n, n), 1.0 / n, recon=recon, riemann=riemann)
    cpu.U[:] = U
    dev = gpu_state(U, (n, n, n), recon=recon, riemann=riemann)
    corr_h = corrections(n ** 3, 7, U[8])
    corr_d = torch.from_numpy(corr_h.ravel().copy()).cuda()
    dt, speed = cpu.compute_dt(0.08)
    decay = float(np.exp(f32(-f32(0.18) * f32(speed) * f32(dt)) / f32(1.0 / n)))
    for _ in range(3):
        cpu.step_radiation(dt, 0.05, corr_h, ch=speed, decay=decay, **flags)
        corr_h[0] = cpu.U[8]  # the driver refreshes slot 0 with the new psi before a step
        pmfmhd.step_cube_radiation(dev, float(dt), float(speed), decay, 0.05, corr_d, **flags)
        corr_d[: n ** 3].copy_(dev.U[8])
    assert not within_parity(cpu.U, pmfmhd.fields_to_host(dev))
    corr_parity(corr_d.cpu().numpy().reshape(9, -1), corr_h)


@pytest.mark.parametrize("track_magnetic", [False, True])
def test_ct_radiation_matches_oracle(track_magnetic):
    n = 16
    dev = gpu_state(problems.smooth_fields(n), (n, n, n), riemann="hlld", mhd_solver="ct")
    pmfmhd.ct_faces_from_cells(dev)
    cpu = oracle.OracleState((n, n, n), 1.0 / n, riemann="hlld", mhd_solver="ct")
    cpu.U[:] = pmfmhd.fields_to_host(dev)
    cpu.faces[:] = dev.ct.packed[: 3 * n ** 3].cpu().numpy().reshape(3, -1)
    corr_h = corrections(n ** 3, 11, 0.0)
    corr_d = torch.from_numpy(corr_h.ravel().copy()).cuda()
    dt, _ = cpu.compute_dt(0.08)
    for _ in range(3):
        cpu.step_radiation(dt, 0.2, corr_h, track_magnetic=track_magnetic)
        pmfmhd.step_ref_radiation(dev, float(dt), 0.0, 1.0, 0.2, corr_d, track_magnetic=track_magnetic)
    host = pmfmhd.fields_to_host(dev)
    assert not within_parity(cpu.U, host)
    faces = dev.ct.packed[: 3 * n ** 3].cpu().numpy().reshape(3, -1)
    for d in range(3):
        assert np.abs(faces[d] - cpu.faces[d]).max() <= 2e-6 + 5e-5 * np.abs(cpu.faces[d]).max()
    rb = dev.ct.packed[18 * n ** 3:].cpu().numpy().reshape(3, -1)
    if track_magnetic:
        assert np.abs(rb - cpu.face_resid).max() <= 1e-6
    else:
        assert np.all(rb == 0)
    corr_parity(corr_d.cpu().numpy().reshape(9, -1), corr_h)
    brms = np.sqrt((host[5:8].astype(np.float64) ** 2).sum() / n ** 3)
    assert pmfmhd.max_divb_face(dev) * dev.dx / brms < 1e-5


def test_zero_correction_untracked_equals_drag_step():
    """With zero corrections and no tracking the radiation kernel is the drag step (to
    rounding: the two instantiations may contract multiply-adds differently)."""
    n = 16
    U = problems.smooth_fields(n)
    a = gpu_state(U, (n, n, n))
    b = gpu_state(U, (n, n, n))
    corr = pmfmhd.allocate_radiation_correction(b)
    dt, speed = pmfmhd.compute_dt(a, 0.08)
    T = f32
    decay = float(np.exp(T(T(-T(0.18) * T(speed) * T(dt)) / T(1.0 / n))))
    for _ in range(3):
        pmfmhd.step_ref_drag(a, float(dt), float(speed), decay, 0.05)
        pmfmhd.step_ref_radiation(b, float(dt), float(speed), decay, 0.05, corr, track_density=False,
                                  track_magnetic=False, track_energy=False)
        corr[: n ** 3].copy_(b.U[8])
    ha, hb = pmfmhd.fields_to_host(a), pmfmhd.fields_to_host(b)
    for v in range(9):
        assert np.abs(ha[v] - hb[v]).max() <= 1e-7 + 2e-6 * np.abs(ha[v]).max(), v
    assert torch.count_nonzero(corr[n ** 3:]) == 0


@pytest.mark.parametrize("mode", ["check", "robust", "global"])
def test_admissibility_flag_and_fallbacks_match_oracle(mode):
    """A low-density pocket stepped with the bulk's dt (the pocket runs far above CFL 1):
    the admissibility check flags exactly the same cells (negative density) as the oracle,
    in FP32 and in FP64, under the plain (HLLD), robust (minmod PLM / HLL) and global (LLF)
    schemes, and every other cell matches the oracle."""
    dims = (24, 12, 10)
    U = problems.turb_field(dims, 1.0 / 24)
    bulk = oracle.OracleState(dims, 1.0 / 24)
    bulk.U[:] = U
    dt, _ = bulk.compute_dt(0.4)
    i, j, k = problems.cell_coords(dims)
    pocket = ((i - 12) ** 2 + (j - 6) ** 2 + (k - 5) ** 2) < 9
    U = U.astype(np.float64)
    U[0, pocket] *= 1e-3
    U[1:4, pocket] *= 1e-3
    U = U.astype(f32)
    cpu = oracle.OracleState(dims, 1.0 / 24)
    cpu.U[:] = U
    dev = gpu_state(U, dims)
    kw = dict(check_admissibility=mode in ("check", "robust"), robust_fallback=mode == "robust",
              global_fallback=mode == "global")
    corr_h = corrections(int(np.prod(dims)), 3, U[8], scale=0.0)
    corr_d = torch.from_numpy(corr_h.ravel().copy()).cuda()
    cpu.step_radiation(dt, 0.1, corr_h, ch=1.0, decay=1.0, **kw)
    c64 = oracle.OracleState(dims, 1.0 / 24, dtype=np.float64)
    c64.U[:] = U
    corr_64 = corrections(int(np.prod(dims)), 3, U[8], scale=0.0).astype(np.float64)
    c64.step_radiation(dt, 0.1, corr_64, ch=1.0, decay=1.0, **kw)
    pmfmhd.step_cube_radiation(dev, float(dt), 1.0, 1.0, 0.1, corr_d, **kw)
    host = pmfmhd.fields_to_host(dev)
    flagged_cpu, flagged_dev = cpu.U[0] < 0, host[0] < 0
    assert flagged_cpu.sum() > 0
    assert np.array_equal(flagged_dev, flagged_cpu)
    assert np.array_equal(flagged_dev, c64.U[0] < 0)
    ok = ~(flagged_cpu | flagged_dev)
    assert not within_parity(cpu.U[:, ok], host[:, ok])
    corr_parity(corr_d.cpu().numpy().reshape(9, -1), corr_h)


def test_global_fallback_is_first_order_on_device():
    """The global fallback zeroes every reconstruction offset (CHECK == 3,
    integrator_cube.jl:168-177): PLM and PPM states step to the same result (to FP32 rounding:
    the two instantiations may contract multiply-adds differently)."""
    dims = (24, 12, 10)
    U = problems.turb_field(dims, 1.0 / 24)
    nc = int(np.prod(dims))
    outs = []
    for recon in ("plm", "ppm"):
        dev = gpu_state(U, dims, recon=recon)
        corr = torch.from_numpy(corrections(nc, 5, U[8], scale=0.0).ravel().copy()).cuda()
        pmfmhd.step_cube_radiation(dev, 2e-3, 1.0, 1.0, 0.1, corr, global_fallback=True)
        outs.append(pmfmhd.fields_to_host(dev).astype(np.float64))
    for f in range(8):
        assert np.abs(outs[1][f] - outs[0][f]).max() <= 1e-6 * np.abs(outs[0][f]).max()


def test_radiation_argument_errors():
    n = 8
    s = gpu_state(problems.smooth_fields(n), (n, n, n))
    corr = pmfmhd.allocate_radiation_correction(s)
    with pytest.raises(pmfmhd.PMFMHDError):
        pmfmhd.step_cube_radiation(s, 1e-3, 1.0, 1.0, -1.0, corr)
    with pytest.raises(pmfmhd.PMFMHDError):
        pmfmhd.step_cube_radiation(s, 1e-3, 1.0, 1.0, 0.1, corr[:-1])
    c = gpu_state(problems.ct_smoke_fields(n), (n, n, n), riemann="hll", mhd_solver="ct")
    with pytest.raises(pmfmhd.PMFMHDError):
        pmfmhd.step_cube_radiation(c, 1e-3, 1.0, 1.0, 0.1, pmfmhd.allocate_radiation_correction(c))
    # the masked fallback is a cube-kernel (GLM) mode: a CT state is refused by the C ABI too
    with pytest.raises(pmfmhd.PMFMHDError):
        pmfmhd._step_radiation(c, 1e-3, 0.0, 1.0, 0.1, pmfmhd.allocate_radiation_correction(c),
                               pmfmhd.RAD_MASKED_FALLBACK, "step")
    rho = s.U[0].clone()
    with pytest.raises(pmfmhd.PMFMHDError):  # the mask may not overwrite its own input
        pmfmhd.radiation_fallback_mask(s, rho, out=rho)
    o = gpu_state(problems.smooth_fields(n), (n, n, n), bcs=("outflow", "periodic", "periodic"))
    with pytest.raises(pmfmhd.PMFMHDError):
        pmfmhd.step_ref_radiation(o, 1e-3, 1.0, 1.0, 0.1, pmfmhd.allocate_radiation_correction(o))


def test_guide_field_compensated_ct_known_answer():
    """test/inherited/test_ct.jl:517-567: 2000 FP32 CT steps on a strong guide field with a
    weak oblique perturbation. Without compensation (plain step, radiation kernel with
    track_magnetic=false) the face divergence random-walks far above round-off and the
    perturbation drifts from FP64; with track_magnetic the faces stay divergence-free to
    round-off and follow FP64."""
    N, nsteps = 16, 2000
    A, hyd, B0 = problems.ct_guide_problem(N)
    nc = N ** 3
    g = gpu_state(np.concatenate([hyd, np.zeros((4, nc), f32)]), (N, N, N), mhd_solver="ct")
    pmfmhd.ct_faces_from_potential(g, A[0], A[1], A[2])
    faces = g.ct.packed[: 3 * nc].cpu().numpy().reshape(3, -1) + np.array(B0, f32)[:, None]

    def state():
        s = gpu_state(np.concatenate([hyd, np.zeros((4, nc), f32)]), (N, N, N), riemann="hlld", mhd_solver="ct")
        return pmfmhd.ct_install_faces(s, faces[0], faces[1], faces[2])

    sp, sn, sc = state(), state(), state()
    # the FP64 run: same faces, cell B = face average, E keeps the thermal pressure
    s64 = oracle.OracleState((N, N, N), 1.0 / N, dtype=np.float64, riemann="hlld", mhd_solver="ct")
    F = faces.astype(np.float64).reshape(3, N, N, N)
    s64.faces[:] = F.reshape(3, -1)
    bc = [0.5 * (F[0] + np.roll(F[0], -1, axis=2)), 0.5 * (F[1] + np.roll(F[1], -1, axis=1)),
          0.5 * (F[2] + np.roll(F[2], -1, axis=0))]
    s64.U[:5] = hyd.astype(np.float64)
    s64.U[4] += 0.5 * sum(b.ravel() ** 2 for b in bc)
    for d in range(3):
        s64.U[5 + d] = bc[d].ravel()
    dt, _ = pmfmhd.compute_dt(sp, 0.3)
    dt = float(f32(dt))
    corr = torch.zeros(9 * nc, dtype=torch.float32, device="cuda")

    def brms64(h):
        return np.sqrt(sum((h[v].astype(np.float64) ** 2).sum() for v in (5, 6, 7)) / nc)

    def divn(s):
        return pmfmhd.max_divb_face(s) * s.dx / brms64(pmfmhd.fields_to_host(s))

    b0 = s64.U[5:8].copy()
    div0 = divn(sp)
    for _ in range(nsteps):
        pmfmhd.step(sp, dt, integrator="ref")
        pmfmhd.step_ref_radiation(sn, dt, 0.0, 1.0, 0.0, corr, track_density=False, track_magnetic=False,
                                  track_energy=False)
        pmfmhd.step_ref_radiation(sc, dt, 0.0, 1.0, 0.0, corr, track_density=False, track_magnetic=True,
                                  track_energy=False)
    for _ in range(nsteps):
        s64.step(dt)
    P = np.abs(s64.U[5:8] - b0).max()

    def err(s):
        return np.abs(pmfmhd.fields_to_host(s)[5:8].astype(np.float64) - s64.U[5:8]).max() / P

    dp, dn, dc = divn(sp), divn(sn), divn(sc)
    ep, en, ec = err(sp), err(sn), err(sc)
    assert div0 < 3e-7
    assert dp > 10 * div0 and dn > 10 * div0
    assert dc < 3 * div0
    assert en > 3 * ec and ep > 3 * ec
    assert ec < 0.05
    assert sc.ct.rbx.abs().max().item() <= 2.1e-6
    assert torch.count_nonzero(sn.ct.rbx) == 0 and torch.count_nonzero(sp.ct.rby) == 0
    h = pmfmhd.fields_to_host(sc)
    bxf = sc.ct.bxf.cpu().numpy().reshape(N, N, N)
    assert np.array_equal((f32(0.5) * (bxf + np.roll(bxf, -1, axis=2))).ravel(), h[5])


def _pocket_state():
    """The low-density pocket of the admissibility test, with the bulk's dt."""
    dims = (24, 12, 10)
    U = problems.turb_field(dims, 1.0 / 24)
    bulk = oracle.OracleState(dims, 1.0 / 24)
    bulk.U[:] = U
    dt, _ = bulk.compute_dt(0.4)
    i, j, k = problems.cell_coords(dims)
    pocket = ((i - 12) ** 2 + (j - 6) ** 2 + (k - 5) ** 2) < 9
    U = U.astype(np.float64)
    U[0, pocket] *= 1e-3
    U[1:4, pocket] *= 1e-3
    return dims, U.astype(f32), dt


@pytest.mark.parametrize("robust", [False, True])
@pytest.mark.parametrize("track_density", [True, False])
def test_masked_fallback_matches_oracle(robust, track_density):
    """The masked fallback (fallback=true, CHECK == 2; integrator_cube.jl:68-83,168-171): the
    mask is built from a first checked trial step as the reference's helpers would
    (radiation_coupling.jl:1536-1577), written into slot 4, and the masked step matches the
    oracle's — the flagged cells exactly, the others to the parity gate — in the plain
    (HLLD) and robust (minmod PLM / HLL) schemes, with and without density tracking (which
    accumulates into the mask's own slot)."""
    dims, U, dt = _pocket_state()
    nc = int(np.prod(dims))
    # trial step, checked: rejected cells come back with negative density
    trial = oracle.OracleState(dims, 1.0 / 24)
    trial.U[:] = U
    c0 = corrections(nc, 3, U[8], scale=0.0)
    trial.step_radiation(dt, 0.1, c0, ch=1.0, decay=1.0, check_admissibility=True)
    assert (trial.U[0] < 0).sum() > 0
    mask_h = oracle.fallback_mask(trial.U[0], dims)
    dev_trial = torch.from_numpy(trial.U[0].copy()).cuda()
    dev = gpu_state(U, dims)
    mask_d = pmfmhd.radiation_fallback_mask(dev, dev_trial)
    assert np.array_equal(mask_d.cpu().numpy(), mask_h)
    corr_h = corrections(nc, 3, U[8], scale=0.0)
    corr_h[4] = mask_h
    corr_d = torch.from_numpy(corr_h.ravel().copy()).cuda()
    kw = dict(fallback=True, robust_fallback=robust, track_density=track_density)
    cpu = oracle.OracleState(dims, 1.0 / 24)
    cpu.U[:] = U
    cpu.step_radiation(dt, 0.1, corr_h, ch=1.0, decay=1.0, **kw)
    pmfmhd.step_cube_radiation(dev, float(dt), 1.0, 1.0, 0.1, corr_d, **kw)
    host = pmfmhd.fields_to_host(dev)
    flagged_cpu, flagged_dev = cpu.U[0] < 0, host[0] < 0
    assert np.array_equal(flagged_dev, flagged_cpu)
    ok = ~(flagged_cpu | flagged_dev)
    assert not within_parity(cpu.U[:, ok], host[:, ok])
    corr_parity(corr_d.cpu().numpy().reshape(9, -1), corr_h)


def test_masked_fallback_everywhere_is_the_global_fallback_on_device():
    """Every cell masked gives the global fallback's scheme (piecewise constant, LLF on every
    face, admissibility flag); a mask of zeros gives the checked step. The instantiations
    differ (HLLD with every face sent to LLF, against the LLF kernel), so the comparison is to
    FP32 rounding, and the flags exactly."""
    dims, U, dt = _pocket_state()
    nc = int(np.prod(dims))

    def run(mask, **kw):
        dev = gpu_state(U, dims)
        corr = torch.from_numpy(corrections(nc, 5, U[8], scale=0.0).ravel().copy()).cuda()
        if mask is not None:
            corr[4 * nc: 5 * nc] = mask
        pmfmhd.step_cube_radiation(dev, float(dt), 1.0, 1.0, 0.1, corr, **kw)
        return pmfmhd.fields_to_host(dev).astype(np.float64)

    pairs = [(run(1.0, fallback=True), run(None, global_fallback=True)),
             (run(0.0, fallback=True), run(None, check_admissibility=True))]
    for a, b in pairs:
        assert np.array_equal(a[0] < 0, b[0] < 0)
        ok = (a[0] > 0) & (b[0] > 0)
        for f in range(8):
            assert np.abs(a[f, ok] - b[f, ok]).max() <= 1e-6 * np.abs(b[f]).max(), f


def test_fallback_mask_matches_oracle():
    """pmfmhd_radiation_fallback_mask against the numpy restatement, the first mask and the
    expanded one, on a non-cubic periodic box."""
    dims = (20, 12, 9)
    nc = int(np.prod(dims))
    rng = np.random.default_rng(11)
    rho = np.where(rng.random(nc) < 0.03, -1.0, 1.0).astype(f32)
    prev = (rng.random(nc) < 0.02).astype(f32)
    s = gpu_state(np.ones((9, nc), f32), dims)  # only the grid matters here
    r = torch.from_numpy(rho).cuda()
    m = torch.from_numpy(prev).cuda()
    assert np.array_equal(pmfmhd.radiation_fallback_mask(s, r).cpu().numpy(), oracle.fallback_mask(rho, dims))
    assert np.array_equal(pmfmhd.radiation_fallback_mask(s, r, m).cpu().numpy(),
                          oracle.fallback_mask(rho, dims, prev))
