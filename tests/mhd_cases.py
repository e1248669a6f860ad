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
