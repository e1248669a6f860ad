"""The radiation step's global fallback in the oracle (CPU): integrator_cube.jl:524-529 launches
it with CHECK == 3, which zeroes the reconstruction offsets of every cell
(integrator_cube.jl:168-177) — piecewise-constant states into LLF, with the admissibility
test. The result therefore cannot depend on the reconstruction the state asks for, and is
not LLF on reconstructed states."""
import numpy as np

import oracle
import problems

f32 = np.float32
DIMS = (24, 12, 10)


def _pocket_field():
    U = problems.turb_field(DIMS, 1.0 / 24)
    bulk = oracle.OracleState(DIMS, 1.0 / 24)
    bulk.U[:] = U
    dt, _ = bulk.compute_dt(0.4)
    i, j, k = problems.cell_coords(DIMS)
    pocket = ((i - 12) ** 2 + (j - 6) ** 2 + (k - 5) ** 2) < 9
    U = U.astype(np.float64)
    U[0, pocket] *= 1e-3
    U[1:4, pocket] *= 1e-3
    return U.astype(f32), dt


def _step(U, dt, recon="plm", riemann="hlld", **kw):
    cpu = oracle.OracleState(DIMS, 1.0 / 24, recon=recon, riemann=riemann)
    cpu.U[:] = U
    corr = np.zeros((9, int(np.prod(DIMS))), f32)
    corr[0] = U[8]
    cpu.step_radiation(dt, 0.1, corr, ch=1.0, decay=1.0, **kw)
    return cpu.U.copy()


def test_global_fallback_is_first_order_llf():
    U, dt = _pocket_field()
    ref = _step(U, dt, global_fallback=True)
    assert (ref[0] < 0).sum() > 0  # the pocket is flagged by the admissibility test
    for recon in ("ppm", "plm_minmod"):
        assert np.array_equal(_step(U, dt, recon=recon, global_fallback=True), ref)
    llf_reconstructed = _step(U, dt, riemann="llf", check_admissibility=True)
    ok = (ref[0] > 0) & (llf_reconstructed[0] > 0)
    assert np.abs(llf_reconstructed[:8, ok] - ref[:8, ok]).max() > 1e-4


# ---- the masked fallback (fallback=true: CHECK == 2, integrator_cube.jl:68-83,168-171,527) ----

def _masked(U, dt, mask, riemann="hlld", recon="plm", track_density=True, **kw):
    cpu = oracle.OracleState(DIMS, 1.0 / 24, recon=recon, riemann=riemann)
    cpu.U[:] = U
    corr = np.zeros((9, int(np.prod(DIMS))), f32)
    corr[0] = U[8]
    corr[4] = mask
    cpu.step_radiation(dt, 0.1, corr, ch=1.0, decay=1.0, track_density=track_density, **kw)
    return cpu.U.copy(), corr


def _pocket_mask():
    i, j, k = problems.cell_coords(DIMS)
    return ((((i - 12) ** 2 + (j - 6) ** 2 + (k - 5) ** 2) < 9)).astype(f32).ravel()


def test_masked_fallback_everywhere_is_the_global_fallback():
    """Every cell masked: zero offsets everywhere and LLF on every face, with the admissibility
    flag — the global fallback's scheme, bit for bit."""
    U, dt = _pocket_field()
    nc = int(np.prod(DIMS))
    got, _ = _masked(U, dt, np.ones(nc, f32), fallback=True)
    assert (got[0] < 0).sum() > 0
    assert np.array_equal(got, _step(U, dt, global_fallback=True))


def test_masked_fallback_without_mask_is_the_checked_step():
    U, dt = _pocket_field()
    got, _ = _masked(U, dt, np.zeros(int(np.prod(DIMS)), f32), fallback=True)
    assert np.array_equal(got, _step(U, dt, check_admissibility=True))


def test_masked_fallback_changes_only_the_masked_cells_and_their_neighbours():
    """A cell's update depends on the states of its own faces, i.e. on itself and its six
    face neighbours: outside the mask dilated by one face step the result is the checked
    step's, bit for bit; inside, the masked scheme differs (and is the global fallback's where
    the mask is dilated far enough, checked above)."""
    U, dt = _pocket_field()
    mask = _pocket_mask()
    got, _ = _masked(U, dt, mask, fallback=True)
    plain = _step(U, dt, check_admissibility=True)
    near = oracle.fallback_mask(np.where(mask > 0, -1.0, 1.0).astype(f32), DIMS) > 0
    assert np.array_equal(got[:, ~near], plain[:, ~near])
    assert np.abs(got[:, near] - plain[:, near]).max() > 1e-6


def test_masked_fallback_reads_the_mask_as_it_was_before_the_step():
    """The density increments of the step land in slot 4, where the mask is: the fields do not
    depend on whether they are tracked, and with tracking the slot ends as mask + increments."""
    U, dt = _pocket_field()
    mask = _pocket_mask()
    a, ca = _masked(U, dt, mask, fallback=True, track_density=True)
    b, cb = _masked(U, dt, mask, fallback=True, track_density=False)
    assert np.array_equal(a, b)
    assert np.array_equal(cb[4], mask)
    inc = ca[4] - mask
    assert np.abs(inc).max() > 0


def test_robust_and_masked_fallback_keep_hll_off_the_mask():
    """robust_fallback with fallback: minmod PLM and HLL, masked cells piecewise constant and
    their faces LLF (integrator_cube.jl:524-529): without a mask it is the robust step."""
    U, dt = _pocket_field()
    nc = int(np.prod(DIMS))
    got, _ = _masked(U, dt, np.zeros(nc, f32), fallback=True, robust_fallback=True)
    assert np.array_equal(got, _step(U, dt, check_admissibility=True, robust_fallback=True))
    got_all, _ = _masked(U, dt, np.ones(nc, f32), fallback=True, robust_fallback=True)
    assert np.array_equal(got_all, _step(U, dt, global_fallback=True))


def test_fallback_mask_follows_the_reference_kernels():
    """oracle.fallback_mask against a loop restatement of _radiation_fallback_mask_k! and
    _radiation_expand_fallback_mask_k! (radiation_coupling.jl:1536-1577) on a small box."""
    dims = (5, 4, 3)
    nx, ny, nz = dims
    rng = np.random.default_rng(3)
    rho = np.where(rng.random(nx * ny * nz) < 0.08, -1.0, 1.0).astype(f32)
    prev = (rng.random(nx * ny * nz) < 0.05).astype(f32)

    def ref(rho, prev):
        out = np.zeros(nx * ny * nz, f32)
        for k in range(nz):
            for j in range(ny):
                for i in range(nx):
                    cells = [(i, j, k), ((i - 1) % nx, j, k), ((i + 1) % nx, j, k), (i, (j - 1) % ny, k),
                             (i, (j + 1) % ny, k), (i, j, (k - 1) % nz), (i, j, (k + 1) % nz)]
                    idx = [(c[2] * ny + c[1]) * nx + c[0] for c in cells]
                    bad = any(rho[q] < 0 for q in idx) or (prev is not None and any(prev[q] > 0 for q in idx))
                    out[(k * ny + j) * nx + i] = 1.0 if bad else 0.0
        return out

    assert np.array_equal(oracle.fallback_mask(rho, dims), ref(rho, None))
    assert np.array_equal(oracle.fallback_mask(rho, dims, prev), ref(rho, prev))
