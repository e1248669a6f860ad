#!/usr/bin/env python
"""Throughput of the PMFGLM MHD step on B200: zone-updates/s of the fused GLM-HLLD step on
a 256^3 FP32 periodic box (seeded turbulent field, MC-PLM, HLLD, CFL 0.2, fixed dt as in
the reference's scripts/benchmark.jl), with roofline, CPU-baseline, end-to-end and clock
records. Prints one JSON line (rank 0).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--n 256]

Multi-GPU runs (torchrun) are independent replicas of the same box on every rank (weak
scaling; the step has no exchange), timed as the max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "pmf-glm_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import numpy as np  # noqa: E402

METRIC = "zone-updates/s at 256^3 + batched mix vs plain FP32; %HBM roof; Linf err vs FP64"
UNIT = "zone-updates/s"
BYTES_PER_ZONE_GLM = 72  # 9 FP32 fields read + 9 written


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--quick", action="store_true", help="skip the secondary measurements")
    ap.add_argument("--ct-only", action="store_true",
                    help="time only the constrained-transport step of the --n box (for kernel profiling)")
    ap.add_argument("--drag-only", action="store_true",
                    help="time only the drag-coupled GLM step (SRC_DRAG) of the --n box")
    ap.add_argument("--compensated-only", action="store_true",
                    help="time only the compensated GLM step of the --n box (for kernel profiling)")
    ap.add_argument("--batched-only", action="store_true",
                    help="time only the batched 64-box mix (--warmup graph-recording steps, then --steps steps)")
    ap.add_argument("--rows", type=int, default=0,
                    help="pin the step kernel's tile height (owned rows per CTA) instead of autotuning it, "
                         "e.g. for a profiler capture whose launch order must not depend on the autotuner")
    return ap.parse_args()


def compensated_only(args):
    """The compensated GLM step (Kahan remainders of momentum, E and B) on the headline box:
    one JSON line with its device time per step."""
    import torch

    import ics
    import pmfmhd
    n = args.n
    s = pmfmhd.set_fields(pmfmhd.allocate_state((n, n, n), 1.0 / n, compensated=True),
                          ics.turbulent_box(n, seed=0)["U"])
    dt, sp = pmfmhd.compute_dt(s, 0.2)
    decay = float(np.exp(np.float32(np.float32(np.float32(-0.18) * np.float32(sp)) * np.float32(dt)) / np.float32(s.dx)))
    if args.rows:
        pmfmhd.set_tile(s, args.rows, 16)
    else:
        pmfmhd.autotune(s)
    for _ in range(args.warmup):
        pmfmhd.step_cube(s, dt, sp, decay)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a0.record(stream)
    for _ in range(args.steps):
        pmfmhd.step_cube(s, dt, sp, decay)
    a1.record(stream)
    torch.cuda.synchronize()
    ms = a0.elapsed_time(a1) / args.steps
    host = pmfmhd.fields_to_host(s)
    print(json.dumps({"compensated_only": True, "n": n, "steps": args.steps, "ms_per_step": ms,
                      "value": n ** 3 / (ms / 1e3), "unit": UNIT, "tile": list(pmfmhd.get_tile(s)),
                      "finite": bool(np.isfinite(host).all())}))


def drag_only(args):
    """The GLM step with source-coupled linear drag (drag impulse 0.05 per step toward rest) on
    the headline box: one JSON line with its device time per step."""
    import torch

    import ics
    import pmfmhd
    n = args.n
    s = pmfmhd.set_fields(pmfmhd.allocate_state((n, n, n), 1.0 / n), ics.turbulent_box(n, seed=0)["U"])
    dt, sp = pmfmhd.compute_dt(s, 0.2)
    decay = float(np.exp(np.float32(np.float32(np.float32(-0.18) * np.float32(sp)) * np.float32(dt)) / np.float32(s.dx)))
    pmfmhd.autotune(s)
    for _ in range(args.warmup):
        pmfmhd.step_cube_drag(s, dt, sp, decay, 0.05)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a0.record(stream)
    for _ in range(args.steps):
        pmfmhd.step_cube_drag(s, dt, sp, decay, 0.05)
    a1.record(stream)
    torch.cuda.synchronize()
    ms = a0.elapsed_time(a1) / args.steps
    host = pmfmhd.fields_to_host(s)
    print(json.dumps({"drag_only": True, "n": n, "steps": args.steps, "ms_per_step": ms,
                      "value": n ** 3 / (ms / 1e3), "unit": UNIT, "tile": list(pmfmhd.get_tile(s)),
                      "finite": bool(np.isfinite(host).all())}))


def ct_only(args):
    """The CT leg alone (faces from the edge potential, autotuned tile, --warmup then --steps
    steps): one JSON line with its device time per step, for profiling the CT kernels."""
    import torch

    import ics
    import pmfmhd
    n = args.n
    boxc = ics.turbulent_box(n, seed=0, with_ct=True)
    c = pmfmhd.set_fields(pmfmhd.allocate_state((n, n, n), 1.0 / n, mhd_solver="ct"), boxc["U"])
    pmfmhd.ct_faces_from_potential(c, *boxc["A_edge"])
    dtc, _ = pmfmhd.compute_dt(c, 0.2)
    if args.rows:
        pmfmhd.set_tile(c, args.rows, 16)
    else:
        pmfmhd.autotune(c)
    for _ in range(args.warmup):
        pmfmhd.step(c, dtc, integrator="ref")
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a0.record(stream)
    for _ in range(args.steps):
        pmfmhd.step(c, dtc, integrator="ref")
    a1.record(stream)
    torch.cuda.synchronize()
    ms = a0.elapsed_time(a1) / args.steps
    host = pmfmhd.fields_to_host(c)
    print(json.dumps({"ct_only": True, "n": n, "steps": args.steps, "ms_per_step": ms,
                      "value": n ** 3 / (ms / 1e3), "unit": UNIT, "tile": list(pmfmhd.get_tile(c)),
                      "finite": bool(np.isfinite(host).all())}))


def batched_only(args):
    """The batched 64-box mix alone: the boxes of `batched_mix`, tiles autotuned per (N, solver)
    or pinned with --rows, --warmup steps (they record the graphs) then --steps timed steps; one
    JSON line with the device time per batch step."""
    import torch

    import ics
    import pmfmhd
    specs = ics.batch_mix(64)
    states = build_boxes(specs)
    seen = set()
    for s, sp in zip(states, specs):
        key = (sp["n"], sp["ct"])
        if key not in seen:
            if args.rows:
                pmfmhd.set_tile(s, args.rows, 16)
            else:
                pmfmhd.autotune(s)
            seen.add(key)
    b = pmfmhd.Batch(states, cfl=0.2)
    b.step(max(2, args.warmup))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    b.step(args.steps)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    finite = all(np.isfinite(b.current_fields(i)).all() for i in range(len(states)))
    b.close()
    cells = sum(sp["n"] ** 3 for sp in specs)
    print(json.dumps({"batched_only": True, "boxes": len(specs), "cells": cells, "steps": args.steps,
                      "ms_per_step": ms, "value": cells / (ms / 1e3), "unit": UNIT, "finite": bool(finite)}))


def workload_config(n, steps):
    return {"workload": f"GLM-HLLD MC-PLM ideal MHD step, {n}^3 periodic FP32 box, gamma=5/3, CFL 0.2 fixed dt",
            "n": n, "ics": "seeded GRF rho=1+0.1g (k^-2, cut N/4), v rms Mach 0.5, B=curl A (P_B~k^2, kc=16), beta=1",
            "steps": steps, "l2": "inputs larger than L2 (state 9x4xN^3 B = %.0f MB)" % (36 * n ** 3 / 1e6),
            "parallelism": "replicas"}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def issue_roof(n, kernel_ms, clocks, device):
    """The FP32-issue side of the roofline: warp instructions per cell of the step kernel (from
    the committed ncu capture) x cells / kernel time, against what the SMs can issue at the
    sampled median SM clock (one warp instruction per sub-partition per cycle, 4 per SM)."""
    import torch
    tf = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(tf):
        return None
    t = json.load(open(tf))
    wi = t.get("glm_warp_inst_per_cell")
    mhz = (clocks or {}).get("sm_mhz")
    if wi is None or not mhz:
        return None
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    achieved = float(wi) * n ** 3 / (kernel_ms / 1e3)
    peak = sms * 4 * float(mhz) * 1e6
    return {"bound": "fp32_issue", "achieved": achieved, "peak": peak, "unit": "warp-instructions/s",
            "frac": achieved / peak, "warp_inst_per_cell": float(wi), "sm_mhz": float(mhz), "sms": sms}


class ClockSampler:
    """nvidia-smi clock/throttle samples while the GPU is busy."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                                       "-lms", "100", "-i", str(gpu_index)], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.f.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        pw = [float(r[3]) for r in rows if r[3].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip() == "Active"})
        load = [s for s, p in zip(sm, pw) if p > 300] or sm
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows), "samples_under_load": len(load)}


def host_cores():
    return int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))


def _oracle_rate(U, n, steps):
    """Zone-updates/s of the oracle FP32 :ref scheme on the n^3 state U (one untimed step,
    then `steps` timed ones)."""
    import oracle
    s = oracle.OracleState((n, n, n), 1 / n, dtype=np.float32)
    s.U[:] = U
    dt, sp = s.compute_dt(0.2)
    s.step(dt, ch=sp)
    t0 = time.perf_counter()
    for _ in range(steps):
        s.step(dt, ch=sp)
    el = time.perf_counter() - t0
    return n ** 3 * steps / el, el


def cpu_baseline(U256):
    """The oracle (C++ restatement of the reference's per-cell :ref scheme, the reference's CPU
    default integrator), FP32, all host threads, on 64^3, 128^3 and the headline 256^3 box of
    the same generator: bounded samples of the workload; `value` is the 256^3 row."""
    import ics
    rows = []
    for n, steps in ((64, 6), (128, 2)):
        v, el = _oracle_rate(ics.turbulent_box(n, seed=0)["U"], n, steps)
        rows.append({"n": n, "steps": steps, "seconds": round(el, 2), "value": v})
    v, el = _oracle_rate(U256, 256, 1)
    rows.append({"n": 256, "steps": 1, "seconds": round(el, 2), "value": v})
    return {"value": v, "unit": UNIT, "cores": host_cores(), "kind": "port",
            "sample": f"oracle FP32 :ref scheme on the 256^3 headline box, 1 step ({el:.1f} s) after one untimed "
                      "step; rows: 64^3, 128^3, 256^3 of the same generator",
            "rows": rows}


REFERENCE_BUDGET_S = 150.0  # wall time the reference arm may spend in warm-up and timed steps


def run_reference(args):
    """The reference arm: the reference's CPU scheme (the oracle's FP32 restatement of the
    per-cell :ref integrator; the reference is Julia, which this image cannot run) on the
    headline box, all host threads. Each step is a full step of the --n box when warm-up and
    timed steps fit REFERENCE_BUDGET_S at the rate of a first probe step; otherwise each step
    is a bounded sample, the same z-slab of that box every step (zone-updates counted over the
    slab). Under torchrun only rank 0 runs."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import ics
    import oracle
    n = args.n
    s = oracle.OracleState((n, n, n), 1 / n, dtype=np.float32)
    s.U[:] = ics.turbulent_box(n, seed=0)["U"]
    dt, sp = s.compute_dt(0.2)
    t0 = time.perf_counter()
    s.step_planes(dt, sp, 0, max(1, n // 16))  # probe: the rate of the scheme on this box
    probe = (time.perf_counter() - t0) / max(1, n // 16) * n  # seconds per full step
    total = args.steps + args.warmup
    planes = n if probe * total <= REFERENCE_BUDGET_S else max(1, int(n * REFERENCE_BUDGET_S / (probe * total)))
    z0 = (n - planes) // 2
    for _ in range(args.warmup):
        s.step_planes(dt, sp, z0, z0 + planes)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        s.step_planes(dt, sp, z0, z0 + planes)
    el = time.perf_counter() - t0
    value = n * n * planes * args.steps / el
    sample = (f"each step: oracle FP32 :ref scheme (the reference's CPU integrator restated in C++; the reference "
              f"is Julia and cannot run here) on the {n}^3 headline box, " +
              ("the full box" if planes == n else f"a {planes}-plane z-slab of it (bounded sample)"))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(args.n, args.steps),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": host_cores(), "kind": "port", "sample": sample,
                             "planes_per_step": planes},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def linf_vs_fp64(n=64, steps=20):
    """Config-0 accuracy: GPU FP32 (plain and compensated) against the FP64 oracle after
    `steps` steps, per field relative to max|field| (L-inf, 99.9th percentile, mean and the
    fraction of cells beyond 1e-5), the FP32 oracle (the reference scheme in FP32) beside it,
    and the energy-ledger drift, in both HLLD degeneracy modes (each against the oracle of the
    same mode), with the device census of near-degenerate HLLD sides over the run. HLL on the
    same box is the control without HLLD's near-degenerate star states."""
    import ics
    import oracle
    import pmfmhd
    box = ics.turbulent_box(n, seed=0)
    U = box["U"]

    def stats(h, ref):
        d = [np.abs(h[v].astype(np.float64) - ref[v]) / max(np.abs(ref[v]).max(), 1e-300) for v in range(8)]
        return {"linf_rel_per_field": [float("%.3e" % x.max()) for x in d],
                "linf_rel_max": float(max(x.max() for x in d)),
                "p999_rel_max": float(max(np.quantile(x, 0.999) for x in d)),
                "mean_rel_max": float(max(x.mean() for x in d)),
                "frac_beyond_1e-5_max": float(max((x > 1e-5).mean() for x in d))}

    out = {"case": f"{n}^3 turbulent box, {steps} steps, CFL 0.2 fixed dt, MC-PLM; FP64 oracle of the same mode as truth"}
    modes = {"relative": pmfmhd.HLLD_DTOL_RELATIVE, "reference": pmfmhd.HLLD_DTOL_REFERENCE}
    truth = {}
    for rs, mode in (("hlld", "relative"), ("hlld", "reference"), ("hll", "relative")):
        tol = modes[mode]
        ref = oracle.OracleState((n, n, n), 1 / n, dtype=np.float64, riemann=rs, hlld_dtol_rel=tol)
        ref.U[:] = U.astype(np.float64)
        dt, sp = ref.compute_dt(0.2)
        e0 = ref.conserved_totals()["energy"]
        o32 = oracle.OracleState((n, n, n), 1 / n, dtype=np.float32, riemann=rs, hlld_dtol_rel=tol)
        o32.U[:] = U
        for _ in range(steps):
            ref.step(dt, ch=sp)
            o32.step(dt, ch=sp)
        truth[(rs, mode)] = ref.U.copy()
        res = {"oracle_fp32": stats(o32.U, ref.U)}
        for comp in (False, True):
            s = pmfmhd.set_fields(pmfmhd.allocate_state((n, n, n), 1 / n, riemann=rs, compensated=comp,
                                                        hlld_dtol_rel=tol), U)
            census = {"solves": 0, "ref_sides": 0, "rel_sides": 0}
            for _ in range(steps):
                if rs == "hlld" and not comp:
                    T = np.float32
                    decay = float(np.exp(T(T(-T(0.18) * T(sp) * T(dt)) / T(s.dx))))
                    c = pmfmhd.step_census(s, float(dt), float(sp), decay)
                    for k in census:
                        census[k] += c[k]
                else:
                    pmfmhd.step(s, float(dt), ch=float(sp))
            r = stats(pmfmhd.fields_to_host(s), ref.U)
            r["energy_ledger_drift"] = abs(pmfmhd.conserved_totals(s)["energy"] - e0) / abs(e0)
            if rs == "hlld" and not comp:
                r["census"] = census
            res["compensated" if comp else "plain"] = r
        out[rs if rs == "hll" else f"hlld_{mode}"] = res
    a, b = truth[("hlld", "reference")], truth[("hlld", "relative")]
    out["fp64_modes_linf_rel_max"] = float(max(np.abs(a[v] - b[v]).max() / np.abs(a[v]).max() for v in range(8)))
    return out


def _field_stats(h, ref):
    d = [np.abs(h[v].astype(np.float64) - ref[v]) / max(np.abs(ref[v]).max(), 1e-300) for v in range(8)]
    return {"linf_rel_max": float(max(x.max() for x in d)), "p999_rel_max": float(max(np.quantile(x, 0.999) for x in d)),
            "mean_rel_max": float(max(x.mean() for x in d))}


def _accuracy_128(U, steps, label):
    """GPU FP32 (plain and compensated) against the FP64 oracle on a 128^3 box, with the
    oracle's own CFL dt sequence replayed on the GPU (so only arithmetic differs)."""
    import oracle
    import pmfmhd
    n = int(round(U.shape[1] ** (1 / 3)))
    ref = oracle.OracleState((n, n, n), 1 / n, dtype=np.float64)
    ref.U[:] = U.astype(np.float64)
    e0 = ref.conserved_totals()["energy"]
    seq = []
    for _ in range(steps):
        dt, sp = ref.compute_dt(0.2)
        ch = float(sp)
        dte = float(dt) * float(sp) / max(float(sp), ch)
        seq.append((dte, ch))
        ref.step(dte, ch=ch)
    out = {"case": label, "steps": steps, "n": n}
    for comp in (False, True):
        s = pmfmhd.set_fields(pmfmhd.allocate_state((n, n, n), 1 / n, compensated=comp), U)
        for dte, ch in seq:
            pmfmhd.step(s, dte, ch=ch)
        h = pmfmhd.fields_to_host(s)
        r = _field_stats(h, ref.U)
        r["energy_ledger_drift"] = abs(pmfmhd.conserved_totals(s)["energy"] - e0) / abs(e0)
        r["finite"] = bool(np.isfinite(h).all())
        out["compensated" if comp else "plain"] = r
        del s
    return out


def big_box_cases():
    """The 512^3 configurations: precision form (plain vs compensated GLM, 20 fixed-dt steps,
    FP64 ledger) and the stress case (Mach 3, beta 0.1, lognormal density with sigma 1,
    P_B ~ k^2 cut at N/8; 40 compensated steps with the on-device CFL of the batch driver),
    each with its FP64-oracle accuracy on 128^3 (the precision form's generator at 128^3;
    the stress box averaged 4^3 -> 128^3)."""
    import torch

    import ics
    import pmfmhd
    n = 512
    out = {}
    box = ics.turbulent_box(n, seed=0)
    U = box["U"]
    del box
    prec = {}
    for comp in (False, True):
        s = pmfmhd.set_fields(pmfmhd.allocate_state((n, n, n), 1 / n, compensated=comp), U)
        pmfmhd.autotune(s)
        pmfmhd.set_fields(s, U)
        if comp:
            for r in s.resid:
                r.zero_()
        e0 = pmfmhd.conserved_totals(s)["energy"]
        dt, sp = pmfmhd.compute_dt(s, 0.2)
        T = np.float32
        decay = float(np.exp(T(T(-T(0.18) * T(sp) * T(dt)) / T(1 / n))))
        pmfmhd.step_cube(s, dt, sp, decay)
        torch.cuda.synchronize()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record()
        for _ in range(20):
            pmfmhd.step_cube(s, dt, sp, decay)
        a1.record()
        torch.cuda.synchronize()
        ms = a0.elapsed_time(a1) / 20
        prec["compensated" if comp else "plain"] = {
            "value": n ** 3 / (ms / 1e3), "ms_per_step": ms,
            "energy_ledger_drift_21_steps": abs(pmfmhd.conserved_totals(s)["energy"] - e0) / abs(e0)}
        del s
        torch.cuda.empty_cache()
    del U
    prec["accuracy_128"] = _accuracy_128(ics.turbulent_box(128, seed=0)["U"], 20, "precision-form generator at 128^3")
    out["precision_512"] = prec
    box = ics.turbulent_box(n, seed=0, mach=3.0, beta=0.1, rho_sigma=1.0, lognormal=True, kc=n / 8)
    U = box["U"]
    del box
    s = pmfmhd.set_fields(pmfmhd.allocate_state((n, n, n), 1 / n, compensated=True), U)
    pmfmhd.autotune(s)
    pmfmhd.set_fields(s, U)
    for r in s.resid:
        r.zero_()
    e0 = pmfmhd.conserved_totals(s)["energy"]
    b = pmfmhd.Batch([s], cfl=0.2)
    torch.cuda.synchronize()
    a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a0.record()
    b.step(40)
    a1.record()
    torch.cuda.synchronize()
    ms = a0.elapsed_time(a1)
    t, _, _ = b.query()
    h = b.current_fields(0)
    b.close()
    brms = float(np.sqrt((h[5:8].astype(np.float64) ** 2).sum() / n ** 3))
    stress = {"value": 40 * n ** 3 / (ms / 1e3), "ms_per_step": ms / 40, "t_end": float(t[0]),
              "finite": bool(np.isfinite(h).all()), "rho_min": float(h[0].min()),
              "energy_ledger_drift": abs(pmfmhd.conserved_totals(s)["energy"] - e0) / abs(e0)}
    s2 = pmfmhd.set_fields(pmfmhd.allocate_state((n, n, n), 1 / n), h)
    stress["divb_centred_dx_over_brms"] = pmfmhd.max_divb(s2) / n / brms
    del s, s2, h
    torch.cuda.empty_cache()
    Ud = U.astype(np.float64).reshape(9, 128, 4, 128, 4, 128, 4).mean(axis=(2, 4, 6)).reshape(9, -1).astype(np.float32)
    del U
    stress["accuracy_128"] = _accuracy_128(Ud, 40, "stress box averaged 4^3 -> 128^3")
    out["stress_512"] = stress
    return out


def plain_port(s, U_host, dt, sp, decay, steps, warmup, entry="pmfport_step_glm"):
    """The plain single-instance FP32 port (pmf-glm_b200/libpmfport.so: one thread per cell,
    the reference's per-cell kernel with its seven Hancock predictions and six Riemann solves per
    cell) on the same state and fixed dt: device ms per step. `entry` pmfport_step_glm shares the
    library's arithmetic; pmfport_step_glm_refarith has the reference's scalar forms."""
    import ctypes

    import torch

    import pmfmhd
    L = ctypes.CDLL(os.path.join(ROOT, "pmf-glm_b200", "libpmfport.so"))
    fn = getattr(L, entry)
    fn.argtypes = [ctypes.POINTER(pmfmhd.Grid), pmfmhd._P9, pmfmhd._P9, ctypes.c_float, ctypes.c_float,
                   ctypes.c_float, ctypes.c_void_p]
    pmfmhd.set_fields(s, U_host)

    def one():
        rc = fn(ctypes.byref(s.grid), pmfmhd._p9(s.U), pmfmhd._p9(s.scratch), float(dt), float(sp), float(decay),
                pmfmhd._stream())
        if rc != 0:
            raise RuntimeError(f"{entry}: {rc}")
        s.U, s.scratch = s.scratch, s.U
    for _ in range(warmup):
        one()
    torch.cuda.synchronize()
    a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a0.record()
    for _ in range(steps):
        one()
    a1.record()
    torch.cuda.synchronize()
    return a0.elapsed_time(a1) / steps


def census_run(s, U_host, dt, sp, decay, steps):
    """HLLD census over `steps` fixed-dt steps of the state's grid from U_host."""
    import pmfmhd
    pmfmhd.set_fields(s, U_host)
    tot = {"solves": 0, "ref_sides": 0, "rel_sides": 0}
    per_step = []
    for _ in range(steps):
        c = pmfmhd.step_census(s, dt, sp, decay)
        per_step.append(c["ref_sides"] + c["rel_sides"])
        for k in tot:
            tot[k] += c[k]
    tot["near_degenerate_sides_per_step"] = per_step
    return tot


def build_boxes(specs):
    """Device states of the batched workload's boxes (host ICs from the seeded generator)."""
    import ics
    import pmfmhd
    states = []
    for sp in specs:
        n = sp["n"]
        b = ics.turbulent_box(n, seed=sp["seed"], beta=sp["beta"], b_index=sp["b_index"], kc=sp["kc"],
                              with_ct=sp["ct"])
        s = pmfmhd.set_fields(pmfmhd.allocate_state((n, n, n), 1.0 / n, mhd_solver="ct" if sp["ct"] else "glm"),
                              b["U"])
        if sp["ct"]:
            pmfmhd.ct_faces_from_potential(s, *b["A_edge"])
        states.append(s)
    return states


def sharded_batched_mix(rank, world, steps=30, nbox=64):
    """The batched workload on `world` GPUs: boxes placed by LPT on N^3 x steps (sharding.py),
    one batch per rank, no collective in the step; value = all zone-updates / max-over-ranks
    device time. Every rank takes the same collective calls."""
    import torch
    import torch.distributed as dist

    import ics
    import pmfmhd
    import sharding
    specs = ics.batch_mix(nbox)
    costs = [sp["n"] ** 3 * steps for sp in specs]
    mine = [specs[i] for i in sharding.lpt_shard(costs, world)[rank]]
    states = build_boxes(mine)
    ms, finite = 0.0, True
    b = pmfmhd.Batch(states, cfl=0.2) if states else None
    if b is not None:
        b.step(2)  # records the graphs
    dist.barrier()
    torch.cuda.synchronize()
    if b is not None:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        b.step(steps)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        finite = all(np.isfinite(b.current_fields(i)).all() for i in range(len(states)))
        b.close()
    t = torch.tensor([ms, 0.0 if finite else 1.0], device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return {"value": sum(costs) / (float(t[0]) / 1e3), "unit": "zone-updates/s", "ranks": world,
            "boxes": nbox, "steps": steps, "placement": "LPT on N^3 x steps", "max_rank_ms": float(t[0]),
            "finite": bool(t[1] == 0)}


def batched_mix(steps=30, nbox=64):
    """Batched form: `nbox` independent periodic boxes of uneven sizes (GLM and CT mixed),
    `steps` steps each with per-box CFL, in one graph-recorded persistent launch per solver
    family per step, against the same boxes advanced one at a time through the plain
    single-box API (compute_dt + step per box per step, the reference's `evolve!` loop)."""
    import torch

    import ics
    import pmfmhd
    specs = ics.batch_mix(nbox)

    states = build_boxes(specs)
    # tiles per N and solver: the autotuner's choice on one box of each kind
    seen = set()
    for s, sp in zip(states, specs):
        key = (sp["n"], sp["ct"])
        if key not in seen:
            pmfmhd.autotune(s)
            seen.add(key)
    host0 = [torch.stack(s.U).clone() for s in states]
    packed0 = [s.ct.packed.clone() if s.ct is not None else None for s in states]
    zones = sum(sp["n"] ** 3 for sp in specs) * steps
    # sequential: one box at a time, host CFL each step
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for s in states:
        for _ in range(steps):
            dt, smax = pmfmhd.compute_dt(s, 0.2)
            if s.ct is not None:
                pmfmhd.step(s, dt, integrator="ref")
            else:
                ch = np.float32(smax)
                pmfmhd.step(s, float(dt) * float(smax) / float(max(np.float32(smax), ch)), ch=float(ch))
    torch.cuda.synchronize()
    seq = time.perf_counter() - t0
    # batched: reset the states, warm (records the two graphs), reset again, time
    def reset():
        for s, u, pk in zip(states, host0, packed0):
            for v in range(9):
                s.U[v].copy_(u[v])
            if pk is not None:
                s.ct.packed.copy_(pk)
    reset()
    b = pmfmhd.Batch(states, cfl=0.2)
    b.step(2)
    b.close()
    reset()
    b = pmfmhd.Batch(states, cfl=0.2)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    b.step(steps)
    e1.record()
    torch.cuda.synchronize()
    bat = e0.elapsed_time(e1) / 1e3
    t, _, _ = b.query()
    finite = all(np.isfinite(b.current_fields(i)).all() for i in range(len(states)))
    b.close()
    sizes = {}
    for sp in specs:
        sizes[sp["n"]] = sizes.get(sp["n"], 0) + 1
    return {"value": zones / bat, "sequential_value": zones / seq, "speedup_vs_sequential": seq / bat,
            "boxes": nbox, "ct_boxes": sum(sp["ct"] for sp in specs), "sizes": sizes, "steps": steps,
            "zone_updates": zones, "batched_s": bat, "sequential_s": seq, "finite": bool(finite),
            "t_min": float(t.min()), "t_max": float(t.max())}


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.ct_only:
        ct_only(args)
        return
    if args.drag_only:
        drag_only(args)
        return
    if args.compensated_only:
        compensated_only(args)
        return
    if args.batched_only:
        batched_only(args)
        return
    import torch
    import torch.distributed as dist

    import ics
    import pmfmhd

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    n = args.n
    box = ics.turbulent_box(n, seed=0)
    U_host = box["U"]
    s = pmfmhd.set_fields(pmfmhd.allocate_state((n, n, n), 1.0 / n, recon="plm", riemann="hlld"), U_host)
    dt, sp = pmfmhd.compute_dt(s, 0.2)
    decay = float(np.exp(np.float32(np.float32(np.float32(-0.18) * np.float32(sp)) * np.float32(dt)) / np.float32(s.dx)))
    if args.rows:
        pmfmhd.set_tile(s, args.rows, 16)
    else:
        pmfmhd.autotune(s)

    sampler = ClockSampler(local)
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        pmfmhd.step_cube(s, dt, sp, decay)
    torch.cuda.synchronize()
    pmfmhd.set_fields(s, U_host)  # warm-up must not advance the measured initial condition
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for k in range(args.steps):
        ev[k][0].record(stream)
        pmfmhd.step_cube(s, dt, sp, decay)
        ev[k][1].record(stream)
    t_end.record(stream)
    torch.cuda.synchronize()
    total_ms = t_start.elapsed_time(t_end)
    kernel_ms = statistics.mean(a.elapsed_time(b) for a, b in ev)
    if world > 1:
        t = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        dist.barrier()
    ms_per_step = total_ms / args.steps
    value = world * n ** 3 * args.steps / (total_ms / 1e3)
    host_after = pmfmhd.fields_to_host(s)
    brms = float(np.sqrt((host_after[5:8].astype(np.float64) ** 2).sum() / n ** 3))
    divb = pmfmhd.max_divb(s) * s.dx / brms

    extra = {"divb_centred_dx_over_brms": divb, "finite": bool(np.isfinite(host_after).all()),
             "positive_density": bool(host_after[0].min() > 0), "kernel_ms": kernel_ms,
             "hlld_dtol_rel": pmfmhd.HLLD_DTOL_RELATIVE}

    # ---- end to end: host state in, host state out, through the C ABI, every step ----------
    # pmfmhd_step_glm_host: the state lives in pinned host memory; each call copies it in,
    # steps it and copies the new state out, pipelined over z-slabs (PCIe both ways
    # overlapped with the compute). Device-timed on the caller's stream.
    pin_in = torch.from_numpy(U_host).pin_memory()
    pin_out = torch.empty_like(pin_in).pin_memory()
    k_e2e = max(1, min(args.steps, 10))
    pmfmhd.step_cube_host(s, pin_in, pin_out, dt, sp, decay)  # warm: context buffers, tensor maps
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(k_e2e):
        pmfmhd.step_cube_host(s, pin_in, pin_out, dt, sp, decay)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / k_e2e
    if world > 1:
        t = torch.tensor([e2e_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e = {"value": world * n ** 3 / (e2e_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": int(pin_in.numel() * 4),
           "d2h_bytes_per_step": int(pin_out.numel() * 4)}

    if not args.quick:
        # the same box with the reference's own HLLD degeneracy test (hlld_dtol_rel = 0): the
        # same kernel, so the same speed; and the census of near-degenerate HLLD sides of the
        # timed run in both modes (the faces where the modes differ)
        r = pmfmhd.set_fields(pmfmhd.allocate_state((n, n, n), 1.0 / n, hlld_dtol_rel=pmfmhd.HLLD_DTOL_REFERENCE),
                              U_host)
        pmfmhd.autotune(r)
        for _ in range(args.warmup):
            pmfmhd.step_cube(r, dt, sp, decay)
        pmfmhd.set_fields(r, U_host)
        torch.cuda.synchronize()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        for _ in range(args.steps):
            pmfmhd.step_cube(r, dt, sp, decay)
        a1.record(stream)
        torch.cuda.synchronize()
        rm = a0.elapsed_time(a1) / args.steps
        hr = pmfmhd.fields_to_host(r)
        extra["reference_mode"] = {"value": n ** 3 / (rm / 1e3), "ms_per_step": rm,
                                   "finite": bool(np.isfinite(hr).all())}
        extra["census"] = {"steps": args.steps,
                           "relative": census_run(s, U_host, dt, sp, decay, args.steps),
                           "reference": census_run(r, U_host, dt, sp, decay, args.steps)}
        del r, hr
        # the plain single-instance FP32 port of the reference's per-cell kernel, same box
        port_ms = plain_port(s, U_host, dt, sp, decay, min(args.steps, 10), 2)
        ref_ms = plain_port(s, U_host, dt, sp, decay, min(args.steps, 10), 2, "pmfport_step_glm_refarith")
        extra["plain_port"] = {"value": n ** 3 / (port_ms / 1e3), "ms_per_step": port_ms,
                               "fused_speedup": port_ms / kernel_ms,
                               "arithmetic": "the library's (decomposition-only comparison)",
                               "reference_arithmetic": {"value": n ** 3 / (ref_ms / 1e3), "ms_per_step": ref_ms,
                                                        "fused_speedup": ref_ms / kernel_ms}}
        # CT side by side on the same generator (faces from the edge potential)
        boxc = ics.turbulent_box(n, seed=0, with_ct=True)
        c = pmfmhd.set_fields(pmfmhd.allocate_state((n, n, n), 1.0 / n, mhd_solver="ct"), boxc["U"])
        pmfmhd.ct_faces_from_potential(c, *boxc["A_edge"])
        dtc, _ = pmfmhd.compute_dt(c, 0.2)
        pmfmhd.autotune(c)
        for _ in range(args.warmup):
            pmfmhd.step(c, dtc, integrator="ref")
        torch.cuda.synchronize()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        for _ in range(args.steps):
            pmfmhd.step(c, dtc, integrator="ref")
        a1.record(stream)
        torch.cuda.synchronize()
        ct_ms = a0.elapsed_time(a1) / args.steps
        hc = pmfmhd.fields_to_host(c)
        brc = float(np.sqrt((hc[5:8].astype(np.float64) ** 2).sum() / n ** 3))
        extra["ct"] = {"value": n ** 3 / (ct_ms / 1e3), "ms_per_step": ct_ms,
                       "divb_face_dx_over_brms": pmfmhd.max_divb_face(c) * c.dx / brc}
        del c
        # compensated GLM
        q = pmfmhd.set_fields(pmfmhd.allocate_state((n, n, n), 1.0 / n, compensated=True), U_host)
        pmfmhd.autotune(q)
        for _ in range(args.warmup):
            pmfmhd.step_cube(q, dt, sp, decay)
        torch.cuda.synchronize()
        a0.record(stream)
        for _ in range(args.steps):
            pmfmhd.step_cube(q, dt, sp, decay)
        a1.record(stream)
        torch.cuda.synchronize()
        cm = a0.elapsed_time(a1) / args.steps
        extra["compensated"] = {"value": n ** 3 / (cm / 1e3), "ms_per_step": cm}
        extra["plain_port"]["compensated_speedup"] = extra["plain_port"]["ms_per_step"] / cm
        extra["plain_port"]["reference_arithmetic"]["compensated_speedup"] = ref_ms / cm
        del q
        if world == 1:
            extra["batched"] = batched_mix()
            extra["big_boxes"] = big_box_cases()
        else:
            extra["batched_sharded"] = sharded_batched_mix(rank, world)
    clocks = sampler.stop()

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return
    peak, peak_kind = measured_peaks()
    achieved = BYTES_PER_ZONE_GLM * n ** 3 / (kernel_ms / 1e3) / 1e9
    traffic = None
    tf = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tf):
        t = json.load(open(tf))
        if "glm_bytes_per_cell" in t:
            traffic = float(t["glm_bytes_per_cell"]) * n ** 3
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "peak_kind": peak_kind,
            "algorithmic_bytes_per_zone": BYTES_PER_ZONE_GLM}
    issue = issue_roof(n, kernel_ms, clocks, local)
    if issue is not None:
        roof["issue"] = issue
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": workload_config(n, args.steps),
            "roofline": roof, "e2e": e2e, "clocks": clocks, "gpu_launches": args.steps}
    if not args.quick and world == 1:
        line["accuracy"] = linf_vs_fp64()
        line["cpu_baseline"] = cpu_baseline(U_host)
    line["extra"] = extra
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
