"""The benchmark's plain single-instance FP32 port (libpmfport.so: one thread per cell, the
reference's per-cell kernel of integrator_ref.jl:69-160 with its seven Hancock predictions and
six solves per cell) against the CPU oracle, in both of its arithmetics: the library's own and
the reference's scalar forms. The port is a baseline of the benchmark, so it has to compute the
same step: the reference's parity gate (test_backends.jl:65-72) on a smooth and a turbulent box."""
import ctypes
import os

import numpy as np
import pytest
import torch

import ics
import oracle
import pmfmhd
import problems
from mhd_cases import within_parity

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ENTRIES = ["pmfport_step_glm", "pmfport_step_glm_refarith"]
MODES = [pytest.param(pmfmhd.HLLD_DTOL_REFERENCE, id="reference"),
         pytest.param(pmfmhd.HLLD_DTOL_RELATIVE, id="relative")]


def port(entry):
    L = ctypes.CDLL(os.path.join(ROOT, "pmf-glm_b200", "libpmfport.so"))
    fn = getattr(L, entry)
    fn.argtypes = [ctypes.POINTER(pmfmhd.Grid), pmfmhd._P9, pmfmhd._P9, ctypes.c_float, ctypes.c_float,
                   ctypes.c_float, ctypes.c_void_p]
    return fn


@pytest.mark.parametrize("dtol", MODES)
@pytest.mark.parametrize("entry", ENTRIES)
@pytest.mark.parametrize("case", ["smooth16", "turb24"])
def test_plain_port_matches_oracle(case, entry, dtol):
    if case == "smooth16":
        n, steps, cfl = 16, 3, 0.08
        U = problems.smooth_fields(n)
    else:
        n, steps, cfl = 24, 2, 0.2
        U = ics.turbulent_box(n, seed=3)["U"]
    dims = (n, n, n)
    cpu = oracle.OracleState(dims, 1.0 / n, hlld_dtol_rel=dtol)
    cpu.U[:] = U
    s = pmfmhd.set_fields(pmfmhd.allocate_state(dims, 1.0 / n, hlld_dtol_rel=dtol), U)
    dt, ch = cpu.compute_dt(cfl)
    T = np.float32
    decay = T(np.exp(T(-T(oracle.GLM_CR) * T(ch) * T(dt) / T(1.0 / n))))
    fn = port(entry)
    for _ in range(steps):
        cpu.step(dt, ch=ch)
        rc = fn(ctypes.byref(s.grid), pmfmhd._p9(s.U), pmfmhd._p9(s.scratch), float(dt), float(ch), float(decay),
                pmfmhd._stream())
        assert rc == 0
        s.U, s.scratch = s.scratch, s.U
    torch.cuda.synchronize()
    host = pmfmhd.fields_to_host(s)
    assert not within_parity(cpu.U, host)
    assert np.abs(host[1] - U[1]).max() > 1e-7  # the state evolved
