"""pmfmhd_conserved_totals_noalloc: FP64 totals for callers that cannot call cudaMalloc.

Such callers (a host application that owns the device memory pool, a plugin that must not
allocate, code that must not allocate between steps) get totals from a scratch array built
into the library instead of a context. This file is collected last on purpose: if it fails,
a run that stops at the first failure has already run every other test.
"""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest
import torch

import oracle
import pmfmhd
import problems

pytestmark = pytest.mark.gpu


def _call_noalloc(s):
    out = (ctypes.c_double * 8)()
    rc = pmfmhd.lib().pmfmhd_conserved_totals_noalloc(ctypes.byref(s.grid), pmfmhd._p9(s.U), out,
                                                       pmfmhd._stream())
    assert rc == 0, pmfmhd.lib().pmfmhd_strerror(rc)
    return np.array(list(out))


def _call_ctx(s):
    t = pmfmhd.conserved_totals(s)
    return np.array([t[k] for k in ("mass", "momx", "momy", "momz", "energy", "Bx", "By", "Bz")])


def _close(a, b):
    # FP64 sums of FP32 values in different orders: agreement to ~1e-12 of the field scale
    scale = np.maximum(np.abs(b), 1e-300)
    return np.all(np.abs(a - b) <= 1e-12 * np.maximum(scale, 1.0) + 1e-15)


def test_noalloc_totals_match_the_context_entry_point_twice_in_a_row():
    n = 40
    first = pmfmhd.set_fields(pmfmhd.allocate_state((n, n, n), 1.0 / n), problems.turb_field((n, n, n), 1.0 / n))
    second = pmfmhd.set_fields(pmfmhd.allocate_state((48, 20, 12), 1.0 / 48),
                               problems.smooth_fields(1, dtype=np.float32).repeat(48 * 20 * 12, axis=1) * 1.5)
    a1 = _call_noalloc(first)
    assert _close(a1, _call_ctx(first))
    a2 = _call_noalloc(second)  # the shared scratch still holds the first call's partials
    assert _close(a2, _call_ctx(second))
    assert not np.allclose(a1, a2)
    assert np.array_equal(_call_noalloc(first), a1)  # same grid again: same bits


def _oracle_totals(s, U):
    cpu = oracle.OracleState(s.dims, s.dx)
    cpu.U[:] = U
    t = cpu.conserved_totals()
    return np.array([t[k] for k in ("mass", "momx", "momy", "momz", "energy", "Bx", "By", "Bz")])


@pytest.mark.parametrize("dims", [(40, 40, 40), (256, 256, 256)], ids=["40^3", "2^24 cells"])
def test_noalloc_totals_match_the_oracle(dims):
    """Directly against the oracle's FP64 totals (diagnostics.jl:44-55), up to the largest grid
    the static scratch takes: exactly 2^24 cells, every partial-sum slot in use."""
    rng = np.random.default_rng(5)
    nc = int(np.prod(dims))
    U = (rng.standard_normal((9, nc), dtype=np.float32) + np.float32(1.5))
    s = pmfmhd.set_fields(pmfmhd.allocate_state(dims, 1.0 / dims[0]), U)
    # FP64 sums of 2^24 values in two orders (blocks of 256 here, the oracle's OpenMP chunks)
    # agree to ~sqrt(n) ulps; a wrong cell or block would be off by ~1e-7 of the total
    got, want = _call_noalloc(s), _oracle_totals(s, U)
    assert np.all(np.abs(got - want) <= 1e-10 * np.abs(want)), (got, want)
    del s
    torch.cuda.empty_cache()


def test_noalloc_totals_survive_a_device_reset():
    """The scratch address is looked up once per CUDA context: after cudaDeviceReset (a host
    that rebuilds its context) the first call looks it up again, and the totals still match the
    oracle. Runs in a child process without torch, so the reset ends no other allocations."""
    r = subprocess.run([sys.executable, os.path.join(os.path.dirname(__file__), "noalloc_reset_child.py")],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr


def test_noalloc_totals_reject_grids_beyond_the_static_scratch():
    g = pmfmhd.Grid(257, 256, 256, (ctypes.c_int32 * 3)(0, 0, 0), 0, 0, 1 / 256, 5 / 3, 1e-6, 1e-7, 1e-4, 0.0, 1e-5)
    fake = pmfmhd._P9(*([0x1000] * 9))  # rejected on the host before any device access
    out = (ctypes.c_double * 8)()
    assert pmfmhd.lib().pmfmhd_conserved_totals_noalloc(ctypes.byref(g), fake, out, None) == -2
    torch.cuda.synchronize()
