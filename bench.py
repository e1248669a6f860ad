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


def cpu_baseline(n=64, steps=6):
    """The oracle (C++ restatement of the reference's per-cell :ref scheme), FP32, all host
    threads, on an n^3 box of the same generator: a bounded sample of the workload."""
    import ics
    import oracle
    box = ics.turbulent_box(n, seed=0)
    s = oracle.OracleState((n, n, n), 1 / n, dtype=np.float32)
    s.U[:] = box["U"]
    dt, sp = s.compute_dt(0.2)
    s.step(dt, ch=sp)  # warm
    t0 = time.perf_counter()
    for _ in range(steps):
        s.step(dt, ch=sp)
    el = time.perf_counter() - t0
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": n ** 3 * steps / el, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"oracle FP32 :ref scheme, {n}^3 box of the same generator, {steps} steps, {el:.1f} s"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import ics
    import oracle
    n = 64
    box = ics.turbulent_box(n, seed=0)
    s = oracle.OracleState((n, n, n), 1 / n, dtype=np.float32)
    s.U[:] = box["U"]
    dt, sp = s.compute_dt(0.2)
    for _ in range(args.warmup):
        s.step(dt, ch=sp)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        s.step(dt, ch=sp)
    el = time.perf_counter() - t0
    value = n ** 3 * args.steps / el
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(args.n, args.steps),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"each step: oracle FP32 :ref scheme on a {n}^3 box of the same generator "
                                       "(the reference is Julia and cannot run here)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def linf_vs_fp64(n=64, steps=20):
    """Config-0 accuracy: GPU FP32 (plain and compensated) against the FP64 oracle after
    `steps` steps, per field relative to max|field| (L-inf, 99.9th percentile and mean), the
    FP32 oracle (the reference scheme in FP32) beside it, and the energy-ledger drift.
    HLL on the same box is the control without HLLD's near-degenerate star states."""
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
                "mean_rel_max": float(max(x.mean() for x in d))}

    out = {"case": f"{n}^3 turbulent box, {steps} steps, CFL 0.2, MC-PLM; FP64 oracle as truth"}
    for rs in ("hlld", "hll"):
        ref = oracle.OracleState((n, n, n), 1 / n, dtype=np.float64, riemann=rs)
        ref.U[:] = U.astype(np.float64)
        dt, sp = ref.compute_dt(0.2)
        e0 = ref.conserved_totals()["energy"]
        o32 = oracle.OracleState((n, n, n), 1 / n, dtype=np.float32, riemann=rs)
        o32.U[:] = U
        for _ in range(steps):
            ref.step(dt, ch=sp)
            o32.step(dt, ch=sp)
        res = {"oracle_fp32": stats(o32.U, ref.U)}
        for comp in (False, True):
            s = pmfmhd.set_fields(pmfmhd.allocate_state((n, n, n), 1 / n, riemann=rs, compensated=comp), U)
            for _ in range(steps):
                pmfmhd.step(s, float(dt), ch=float(sp))
            r = stats(pmfmhd.fields_to_host(s), ref.U)
            r["energy_ledger_drift"] = abs(pmfmhd.conserved_totals(s)["energy"] - e0) / abs(e0)
            res["compensated" if comp else "plain"] = r
        out[rs] = res
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
             "positive_density": bool(host_after[0].min() > 0), "kernel_ms": kernel_ms}

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
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": workload_config(n, args.steps),
            "roofline": roof, "e2e": e2e, "clocks": clocks, "gpu_launches": args.steps}
    if not args.quick and world == 1:
        line["accuracy"] = linf_vs_fp64()
        line["cpu_baseline"] = cpu_baseline()
    line["extra"] = extra
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
