"""Config-0 gate: the seeded 64^3 turbulent box of the benchmark generator (rho = 1 + 0.1 g with
g a k^-2 Gaussian random field cut at N/4; velocity rms Mach 0.5 at c_s = 1; B = curl A with
P_B ~ k^2 cut sharply at k = 16, scaled to beta = 1; psi = 0), MC-PLM, HLLD, gamma 5/3, dt from
CFL 0.2 on the initial state held fixed (the reference's warm loop, scripts/benchmark.jl:53-62),
20 steps, on the GPU through the C ABI, in both HLLD degeneracy modes. Truth is the oracle in
FP64 (the reference's Float64 path) in the same mode; the oracle in FP32 is the reference's
Float32 path.

Tolerances, per field relative to max|field of the reference| (BULK and LINF_FP64 below):
  * mass drift |M/M0 - 1| <= 3e-6 (test/test_backends.jl:118);
  * bulk: 99.9th percentile, mean, and the fraction of cells beyond 1e-5 (the north_star's
    L-inf figure), against FP64 and against FP32;
  * L-inf against FP64 per field: no worse than the reference's own FP32 arithmetic (the FP32
    oracle) is on this box, rounded up.
The scheme's L-inf is set by a handful of HLLD faces whose single-star denominator denK sits
within FP32 rounding of zero (the census counts them: 3 sides in 15.7 M solves over the 20
steps), where the flux is ill-conditioned in its inputs: the reference's FP32 path is 1.8e-3
(relative mode) and 4.7e-2 (the reference's absolute test) from FP64 there, worst field, and
the perturbation of such an event spreads to ~0.04 % of the cells in the absolute mode. The
device measured 2.9e-4 and 4.1e-2. Everywhere else FP32 tracks FP64 to rounding (99.9th
percentile ~2e-7).
"""
import numpy as np
import pytest

import ics
import oracle
import pmfmhd
from mhd_cases import rel_linf

pytestmark = pytest.mark.gpu

N, STEPS = 64, 20
FIELDS = ("rho", "mx", "my", "mz", "E", "Bx", "By", "Bz")
# L-inf against the FP64 oracle of the same mode, per field (rho, mx, my, mz, E, Bx, By, Bz);
# the FP32 oracle measured 1.8e-3 1.0e-3 6.4e-4 1.4e-3 1.3e-3 1.6e-4 4.1e-4 1.0e-3 (relative)
# and 4.3e-2 2.1e-2 1.8e-2 1.6e-2 4.7e-2 2.4e-3 1.4e-2 2.8e-2 (reference)
LINF_FP64 = {
    "relative": (2e-3, 1e-3, 7e-4, 1.5e-3, 1.5e-3, 2e-4, 5e-4, 1.1e-3),
    "reference": (5e-2, 2.5e-2, 2e-2, 2e-2, 5e-2, 3e-3, 2e-2, 3e-2),
}
# bulk bounds: (p99.9 vs FP64, mean vs FP64, fraction beyond 1e-5 vs FP64, p99.9 vs FP32,
# mean vs FP32); measured 2.2e-7 4.0e-8 1.0e-4 8.1e-7 6.4e-8 (relative) and
# 6.2e-7 4.8e-7 3.9e-4 7.5e-6 8.5e-7 (reference)
BULK = {
    "relative": (1e-6, 1e-7, 5e-4, 2e-6, 2e-7),
    "reference": (2e-6, 1e-6, 1e-3, 2e-5, 2e-6),
}
MODES = {"relative": pmfmhd.HLLD_DTOL_RELATIVE, "reference": pmfmhd.HLLD_DTOL_REFERENCE}

_cache = {}


def _box():
    if "U" not in _cache:
        _cache["U"] = ics.turbulent_box(N, seed=0)["U"]
    return _cache["U"]


def _oracle_run(mode, dtype):
    key = (mode, np.dtype(dtype).name)
    if key not in _cache:
        s = oracle.OracleState((N,) * 3, 1 / N, dtype=dtype, hlld_dtol_rel=MODES[mode])
        s.U[:] = _box()
        dt, sp = _oracle_dt()
        for _ in range(STEPS):
            s.step(dt, ch=sp)
        _cache[key] = s.U.copy()
    return _cache[key]


def _oracle_dt():
    s = oracle.OracleState((N,) * 3, 1 / N, dtype=np.float64)
    s.U[:] = _box()
    return s.compute_dt(0.2)


def _stats(cand, ref):
    out = {"linf": [], "p999": [], "mean": [], "beyond_1e-5": []}
    for v in range(8):
        r = ref[v].astype(np.float64)
        d = np.abs(cand[v].astype(np.float64) - r) / max(np.abs(r).max(), 1e-300)
        out["linf"].append(float(d.max()))
        out["p999"].append(float(np.quantile(d, 0.999)))
        out["mean"].append(float(d.mean()))
        out["beyond_1e-5"].append(float((d > 1e-5).mean()))
    return out


@pytest.mark.parametrize("mode", ["relative", "reference"])
def test_cfg0_box_against_fp64_and_fp32_oracles(mode):
    U = _box()
    dt, sp = _oracle_dt()
    dev = pmfmhd.set_fields(pmfmhd.allocate_state((N,) * 3, 1 / N, hlld_dtol_rel=MODES[mode]), U)
    T = np.float32
    decay = float(np.exp(T(T(-T(0.18) * T(sp) * T(dt)) / T(dev.dx))))
    census = {"solves": 0, "ref_sides": 0, "rel_sides": 0}
    for _ in range(STEPS):
        c = pmfmhd.step_census(dev, float(dt), float(sp), decay)
        for k in census:
            census[k] += c[k]
    host = pmfmhd.fields_to_host(dev)
    assert np.isfinite(host).all() and host[0].min() > 0
    o64, o32 = _oracle_run(mode, np.float64), _oracle_run(mode, np.float32)
    s64, s32 = _stats(host, o64), _stats(host, o32)
    o32_vs_64 = rel_linf(o32, o64)
    report = {"mode": mode, "census": census, "vs_fp64": s64, "vs_fp32": s32, "oracle_fp32_vs_fp64": o32_vs_64}
    print(report)
    # the near-degenerate sides that set L-inf are few
    assert census["solves"] >= 0.99 * 3 * N ** 3 * STEPS
    assert census["ref_sides"] + census["rel_sides"] <= 50, census
    m0 = U[0].astype(np.float64).sum()
    assert abs(host[0].astype(np.float64).sum() / m0 - 1) <= 3e-6
    p64, m64, b64, p32, m32 = BULK[mode]
    for f, name in enumerate(FIELDS):
        assert s64["p999"][f] <= p64 and s64["mean"][f] <= m64 and s64["beyond_1e-5"][f] <= b64, (name, report)
        assert s32["p999"][f] <= p32 and s32["mean"][f] <= m32, (name, report)
        assert s64["linf"][f] <= LINF_FP64[mode][f], (name, report)
