"""The host-buffer GLM step (pmfmhd_step_glm_host: z-slab pipeline of copy in / step / copy
out) gives the same bits as the device step on every chunking, grid shape and boundary."""
import numpy as np
import pytest
import torch

import pmfmhd
import problems

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dims,bcs", [((32, 32, 32), ("periodic",) * 3), ((37, 11, 20), ("periodic",) * 3),
                                      ((24, 16, 18), ("outflow", "periodic", "reflecting")),
                                      ((32, 16, 96), ("periodic",) * 3),
                                      ((16, 24, 70), ("periodic", "periodic", "outflow"))])
@pytest.mark.parametrize("nchunks", [1, 3, 8])
def test_host_step_equals_device_step(dims, bcs, nchunks):
    U = problems.turb_field(dims, 1.0 / max(dims))
    s = pmfmhd.set_fields(pmfmhd.allocate_state(dims, 1.0 / max(dims), bcs=bcs), U)
    dt, sp = pmfmhd.compute_dt(s, 0.2)
    hin = torch.from_numpy(U.copy()).pin_memory()
    hout = torch.empty_like(hin).pin_memory()
    for _ in range(2):  # a second call reuses the context's buffers
        pmfmhd.step_cube_host(s, hin, hout, float(dt), float(sp), 0.98, nchunks=nchunks)
        smax_host = pmfmhd.last_wavespeed(s)
        pmfmhd.step_cube(s, float(dt), float(sp), 0.98)
        smax_dev = pmfmhd.last_wavespeed(s)
        assert np.array_equal(hout.numpy(), pmfmhd.fields_to_host(s))
        assert smax_host == smax_dev
        hin.copy_(hout)


def test_host_step_with_pageable_memory():
    dims = (32, 24, 16)
    U = problems.turb_field(dims, 1.0 / 32)
    s = pmfmhd.set_fields(pmfmhd.allocate_state(dims, 1.0 / 32), U)
    hin, hout = torch.from_numpy(U.copy()), torch.empty((9, U.shape[1]), dtype=torch.float32)
    pmfmhd.step_cube_host(s, hin, hout, 1e-3, 2.0, 0.99, nchunks=4)
    pmfmhd.step_cube(s, 1e-3, 2.0, 0.99)
    assert np.array_equal(hout.numpy(), pmfmhd.fields_to_host(s))
    with pytest.raises(pmfmhd.PMFMHDError):
        pmfmhd.step_cube_host(s, hin[:8], hout, 1e-3, 2.0, 0.99)
