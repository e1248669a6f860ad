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
