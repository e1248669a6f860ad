"""Shared test drivers: the reference tests' known-answer runs, written once and driven by
either the CPU oracle (OracleState) or the CUDA library (pmfmhd), which expose the same
step / evolve / diagnostics API."""
import json
import os

import numpy as np

import problems

HERE = os.path.dirname(os.path.abspath(__file__))
KNOWN = json.load(open(os.path.join(HERE, "golden", "known_answers.json")))
PAR = KNOWN["parity"]


def within_parity(ref, cand, rtol=PAR["rtol"], atol=PAR["atol"]):
    """Per-field gate of test_backends.jl:65-72: max|cand-ref| <= atol + rtol*max|ref|."""
    bad = []
    for v in range(ref.shape[0]):
        err = float(np.abs(cand[v].astype(np.float64) - ref[v].astype(np.float64)).max())
        lim = atol + rtol * float(np.abs(ref[v]).max())
        if not np.isfinite(cand[v]).all() or err > lim:
            bad.append((v, err, lim))
    return bad


def alfven_L1(make_state, get_fields, totals, evolve, N, amp=0.1, p0=0.1, tfinal=0.5, cfl=0.4, recon="plm",
              glm_cr=0.18):
    """test/inherited/runtests.jl:6-25 on an (N,4,4) box."""
    s = make_state((N, 4, 4), 1.0 / N, recon)
    t0 = totals(s)
    t, n = evolve(s, tfinal, cfl, glm_cr)
    t1 = totals(s)
    By = get_fields(s)[6][:N].astype(np.float64)
    x = (np.arange(1, N + 1) - 0.5) / N
    L1 = float(np.abs(By - problems.alfven_by_exact(x, t, 1.0, amp=amp)).sum() / N)
    drift = {"mass": abs(t1["mass"] - t0["mass"]) / abs(t0["mass"]),
             "energy": abs(t1["energy"] - t0["energy"]) / abs(t0["energy"])}
    return L1, n, t, drift


def near_degenerate_box(dims, delta=1e-3, eps=1e-5, seed=3, gamma=5 / 3):
    """Uniform gas (rho 1, p 0.1) threaded by a unit field along x, so the Alfven speed (1)
    exceeds the sound speed, with small random transverse field (rms `delta`) and velocity
    (rms `eps`). On every x-face the fast and Alfven speeds then nearly coincide and HLLD's
    single-star denominator denK = d(S-u)(S-SM) - bn^2 sits within ~1e-6 bn^2 of zero: the
    faces where the reference's absolute degeneracy test and the relative one differ. Not one
    of the reference's problems; a stress case for glm_physics.jl:255-263."""
    nx, ny, nz = dims
    n = nx * ny * nz
    r = np.random.default_rng(seed)
    rho = np.ones(n)
    p = np.full(n, 0.1)
    v = r.standard_normal((3, n)) * eps
    B = np.zeros((3, n))
    B[0] = 1.0
    B[1] = r.standard_normal(n) * delta
    B[2] = r.standard_normal(n) * delta
    U = np.zeros((9, n))
    U[0] = rho
    U[1:4] = rho * v
    U[4] = p / (gamma - 1) + 0.5 * rho * (v ** 2).sum(0) + 0.5 * (B ** 2).sum(0)
    U[5:8] = B
    return U.astype(np.float32)


def rel_linf(cand, ref, fields=range(8)):
    """Per-field max|cand-ref| / max|ref| (FP64 arithmetic)."""
    out = []
    for v in fields:
        r = np.asarray(ref[v], dtype=np.float64)
        out.append(float(np.abs(np.asarray(cand[v], dtype=np.float64) - r).max() / max(np.abs(r).max(), 1e-300)))
    return out
