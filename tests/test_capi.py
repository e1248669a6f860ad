"""The C-ABI library loads without a GPU and exports every entry point include/pmfmhd.h
declares; argument checks reject bad calls before touching the device."""
import ctypes
import os
import re

import pytest

import pmfmhd

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", f) for f in sorted(os.listdir(os.path.join(ROOT, "include"))) if f.endswith(".h")]


def declared_functions():
    names = []
    for h in HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(pmfmhd_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "pmfmhd_step_glm" in names and "pmfmhd_step_ct" in names and "pmfmhd_max_wavespeed" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(pmfmhd.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_python_mirror_binds_every_declared_symbol():
    assert set(declared_functions()) <= set(pmfmhd.SIGNATURES), set(declared_functions()) - set(pmfmhd.SIGNATURES)


def test_version_and_strerror():
    L = pmfmhd.lib()
    assert L.pmfmhd_version() >= 100
    assert L.pmfmhd_strerror(0) == b"ok"
    assert L.pmfmhd_strerror(-2) == b"invalid grid shape"
    assert L.pmfmhd_strerror(-7) == b"unsupported combination"


def test_null_context_is_rejected_without_device_work():
    L = pmfmhd.lib()
    g = pmfmhd.Grid(8, 8, 8, (ctypes.c_int32 * 3)(0, 0, 0), 0, 0, 0.125, 5 / 3, 1e-6, 1e-7, 1e-4, 0.0)
    p9 = pmfmhd._P9(*([None] * 9))
    assert L.pmfmhd_step_glm(None, ctypes.byref(g), p9, p9, 1e-3, 1.0, 1.0, None, None) == -1
    assert L.pmfmhd_step_ct(None, ctypes.byref(g), p9, p9, None, 1e-3, None, 0, None) == -1
    assert L.pmfmhd_max_wavespeed(None, ctypes.byref(g), p9, None, None) == -1
    assert L.pmfmhd_create(0, None) == -1
    assert L.pmfmhd_destroy(None) == 0


def test_grid_struct_layout_matches_header():
    assert ctypes.sizeof(pmfmhd.Grid) == 4 * 15
    assert pmfmhd.Grid.dx.offset == 32
    assert pmfmhd.Grid.hlld_dtol_rel.offset == 56


@pytest.mark.parametrize("kw,msg", [
    (dict(mhd_solver="bogus"), "unknown mhd_solver"),
    (dict(mhd_solver="ct", bcs=("outflow", "periodic", "periodic")), "periodic"),
    (dict(riemann="roe"), "unknown MHD riemann"),
    (dict(recon="weno"), "unknown recon"),
    (dict(bc="open"), "unknown BC"),
])
def test_allocate_state_rejects_like_the_reference(kw, msg):
    with pytest.raises(pmfmhd.PMFMHDError, match=msg):
        pmfmhd.allocate_state((8, 8, 8), 1 / 8, **kw)
