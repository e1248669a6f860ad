"""Child process of tests/test_zz_no_alloc.py: pmfmhd_conserved_totals_noalloc across a
cudaDeviceReset. Runs without torch: device buffers come from the CUDA runtime that
libpmfmhd.so itself loaded, so the reset ends no one else's allocations. Prints "ok" when the
totals before and after the reset both match the oracle's."""
import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle  # noqa: E402

LIB = ctypes.CDLL(os.path.join(ROOT, "pmf-glm_b200", "libpmfmhd.so"))
RT = ctypes.CDLL("libcudart.so.12")  # the runtime the library was loaded with (same soname)
H2D = 1


class Grid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
                ("bc", ctypes.c_int32 * 3), ("recon", ctypes.c_int32), ("riemann", ctypes.c_int32),
                ("dx", ctypes.c_float), ("gamma", ctypes.c_float), ("smallr", ctypes.c_float),
                ("pfl", ctypes.c_float), ("llf_dmin", ctypes.c_float), ("llf_pmin", ctypes.c_float),
                ("hlld_dtol_rel", ctypes.c_float)]


def ck(rc, what):
    if rc != 0:
        raise SystemExit(f"{what} returned {rc}")


def upload(U):
    ptrs = []
    for f in range(9):
        p = ctypes.c_void_p()
        ck(RT.cudaMalloc(ctypes.byref(p), ctypes.c_size_t(U[f].nbytes)), "cudaMalloc")
        ck(RT.cudaMemcpy(p, U[f].ctypes.data_as(ctypes.c_void_p), ctypes.c_size_t(U[f].nbytes), H2D), "cudaMemcpy")
        ptrs.append(p)
    return ptrs


def totals(grid, ptrs):
    out = (ctypes.c_double * 8)()
    ck(LIB.pmfmhd_conserved_totals_noalloc(ctypes.byref(grid), (ctypes.c_void_p * 9)(*[p.value for p in ptrs]), out,
                                           None), "pmfmhd_conserved_totals_noalloc")
    return np.array(list(out))


def oracle_totals(dims, dx, U):
    s = oracle.OracleState(dims, dx)
    s.U[:] = U
    t = s.conserved_totals()
    return np.array([t[k] for k in ("mass", "momx", "momy", "momz", "energy", "Bx", "By", "Bz")])


def close(a, b):
    return np.all(np.abs(a - b) <= 1e-12 * np.maximum(np.abs(b), 1.0))


def main():
    dims, dx = (40, 24, 18), 1.0 / 40
    grid = Grid(dims[0], dims[1], dims[2], (ctypes.c_int32 * 3)(0, 0, 0), 0, 0, dx, 5 / 3, 1e-6, 1e-7, 1e-4, 0.0,
                1e-5)
    rng = np.random.default_rng(11)
    nc = int(np.prod(dims))
    U1 = (rng.standard_normal((9, nc)) + 2.0).astype(np.float32)
    U2 = (rng.standard_normal((9, nc)) * 3.0 - 1.0).astype(np.float32)
    p1 = upload(U1)
    a1 = totals(grid, p1)  # first call in this context: the address is looked up
    if not close(a1, oracle_totals(dims, dx, U1)):
        raise SystemExit(f"before reset: {a1} != oracle")
    for p in p1:
        RT.cudaFree(p)
    ck(RT.cudaDeviceSynchronize(), "cudaDeviceSynchronize")
    ck(RT.cudaDeviceReset(), "cudaDeviceReset")  # ends this process's context; the module reloads
    p2 = upload(U2)
    a2 = totals(grid, p2)  # a new context: the address is looked up again
    if not close(a2, oracle_totals(dims, dx, U2)):
        raise SystemExit(f"after reset: {a2} != oracle")
    a3 = totals(grid, p2)
    if not np.array_equal(a2, a3):
        raise SystemExit("second call after reset differs")
    for p in p2:
        RT.cudaFree(p)
    print("ok")


if __name__ == "__main__":
    main()
