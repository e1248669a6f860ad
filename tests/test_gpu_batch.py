"""The batched driver (one persistent launch per solver family, on-device per-box CFL)
against the same boxes advanced one by one through the single-box API and the oracle,
with the per-step rule of `evolve!` (driver.jl:48-71): dt = cfl*dx/smax, ch = fac*smax,
dt scaled by smax/max(smax, ch), decay = exp(-cr*ch*dt/dx)."""
import numpy as np
import pytest
import torch

import ics
import oracle
import pmfmhd
from mhd_cases import within_parity

pytestmark = pytest.mark.gpu
f32 = np.float32


def make_box(n, seed, ct, comp=False):
    if ct:
        b = ics.turbulent_box(n, seed=seed, with_ct=True)
        s = pmfmhd.set_fields(pmfmhd.allocate_state((n, n, n), 1.0 / n, mhd_solver="ct", compensated=comp), b["U"])
        pmfmhd.ct_faces_from_potential(s, *b["A_edge"])
    else:
        b = ics.turbulent_box(n, seed=seed)
        s = pmfmhd.set_fields(pmfmhd.allocate_state((n, n, n), 1.0 / n, compensated=comp), b["U"])
    return s


def clone(s):
    c = pmfmhd.allocate_state(s.dims, s.dx, mhd_solver=s.mhd_solver(), compensated=s.resid is not None)
    for v in range(9):
        c.U[v].copy_(s.U[v])
    if s.ct is not None:
        c.ct.packed.copy_(s.ct.packed)
    return c


def evolve_steps(s, nsteps, cfl, fac=1.0, cr=0.18):
    """`evolve!`'s loop body for a fixed number of steps; returns the elapsed time."""
    t = 0.0
    for _ in range(nsteps):
        dt, smax = pmfmhd.compute_dt(s, cfl)
        if pmfmhd.uses_ct(s):
            dtf = float(dt)
            pmfmhd.step(s, dtf, integrator="ref")
        else:
            ch = f32(f32(fac) * f32(smax))
            dtf = float(dt) * float(smax) / float(max(f32(smax), ch))
            pmfmhd.step(s, dtf, ch=float(ch), glm_cr=cr)
        t += dtf
    return t


@pytest.mark.parametrize("nsteps", [1, 4])
def test_batch_matches_per_box_steps(nsteps):
    specs = [(32, 1, False), (48, 2, False), (16, 3, False), (32, 4, True), (24, 5, True), (40, 6, False)]
    boxes = [make_box(n, seed, ct) for n, seed, ct in specs]
    singles = [clone(s) for s in boxes]
    batch = pmfmhd.Batch(boxes, cfl=0.2, glm_ch_fac=1.0, glm_cr=0.18)
    batch.step(nsteps)
    t, par, _ = batch.query()
    assert np.all(par == nsteps % 2)
    for i, (s, ref) in enumerate(zip(boxes, singles)):
        tr = evolve_steps(ref, nsteps, 0.2)
        got = batch.current_fields(i)
        assert not within_parity(pmfmhd.fields_to_host(ref), got), i
        assert abs(t[i] / tr - 1) < 1e-6, (i, t[i], tr)
        if s.ct is not None:
            fb = s.ct.packed[: 3 * s.nc].cpu().numpy()
            fr = ref.ct.packed[: 3 * ref.nc].cpu().numpy()
            assert np.abs(fb - fr).max() <= 2e-6 + 5e-5 * np.abs(fr).max()
    batch.close()


def test_batch_matches_oracle():
    n, steps = 16, 3
    specs = [(n, 11, False), (n, 12, True)]
    boxes = [make_box(m, seed, ct) for m, seed, ct in specs]
    refs = []
    for s in boxes:
        o = oracle.OracleState(s.dims, 1.0 / n, mhd_solver=s.mhd_solver())
        o.U[:] = pmfmhd.fields_to_host(s)
        if s.ct is not None:
            o.faces[:] = s.ct.packed[: 3 * s.nc].cpu().numpy().reshape(3, -1)
        refs.append(o)
    batch = pmfmhd.Batch(boxes, cfl=0.3)
    batch.step(steps)
    for o in refs:
        for _ in range(steps):
            dt, smax = o.compute_dt(0.3)
            if o.mhd_solver == "ct":
                o.step(dt)
            else:
                ch = f32(smax)
                o.step(float(dt) * float(smax) / float(max(smax, ch)), ch=ch)
    for i, o in enumerate(refs):
        assert not within_parity(o.U, batch.current_fields(i)), i
    batch.close()


def test_batch_compensated_and_long_run_stays_finite():
    boxes = [make_box(32, 21, False, comp=True), make_box(32, 22, True, comp=True), make_box(48, 23, False)]
    batch = pmfmhd.Batch(boxes, cfl=0.2)
    batch.step(10)
    t, par, dt = batch.query()
    assert np.all(t > 0) and np.all(dt > 0)
    for i in range(len(boxes)):
        h = batch.current_fields(i)
        assert np.isfinite(h).all() and h[0].min() > 0
    torch.cuda.synchronize()
    batch.close()
