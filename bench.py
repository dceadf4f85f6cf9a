#!/usr/bin/env python
"""Benchmark of the seismod FDTD hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload a3d|a3d512|eiso|eiso1|serve]
                    [--precision fp32|fp16|bf16|fp64]

A "step" is one FDTD time step of the whole workload (velocity + pressure /
stress update, CPML/PML memory variables, source injection, receiver
sampling).  Default workload: the 256^3 a_iso_3d shot (+2x16 CPML = 288^3,
FP32, 16,384 surface receivers).  Inputs (wavefields, materials) stay
resident in HBM; the state (~0.4 GB in FP32) is larger than the 126 MB L2,
so no flush is needed between timed steps.

Prints ONE JSON line (rank 0).  N > 1 (torchrun): every rank runs its own
shot (replicas, no collective in the data path); the time is the max over
ranks; value = all ranks' cell-updates / that time.

--impl reference times the reference's own CPU program (oracle/_ref, built
from its sources) on the host cores for a bounded number of steps of the
same workload.

Every device handle is autotuned (launch configuration) and replays its time
loop as CUDA graphs of 16 steps unless --no-tune / --no-graph.  --workload
eiso adds the batching comparison (plain single-shot FP32 against 64 batched
shots in FP32, FP16 and BF16, trace errors against FP64); --workload serve
runs the mixed Poisson request stream through the request loop and reports
p50/p99 latency beside shots/s and Gcell/s.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import math
import os
import resource
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("shots/s & Gcell/s, batched+FP16 vs plain FP32 (trace err≤1e-3); "
          "HBM %peak; p50/p99")


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            m = json.load(f)
        return float(m["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ----------------------------------------------------------------------------
# clocks sampled during the timed region
# ----------------------------------------------------------------------------

class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.rows = []
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.p = None
        return self

    def _read(self):
        for line in self.p.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.p:
            time.sleep(0.25)
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in self.rows for n, v in zip(names, r[5:9]) if v == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


# ----------------------------------------------------------------------------
# workloads and algorithmic bytes
# ----------------------------------------------------------------------------

# bytes per stored value in block storage: a 16-bit mantissa and the share
# of the block's exponent byte (a_iso_3d: blocks of 4 y rows; e_iso: 4 x rows)
A3D_BFP_BYTES = 2.25
EISO_BFP_BYTES = 2.25


def a3d_bytes_per_step(p, s, m=4, psi=None):
    """Ncell (8 s + 2 m) + sum over axes of N_slab 4 p (state R+W, rho & K read
    once, both CPML memory variables R+W on their slabs).  Block storage:
    s = A3D_BFP_BYTES (a mantissa and a share of an exponent byte per value),
    p = 4 (FP32 memory variables)."""
    psi = s if psi is None else psi
    n2 = [n + 2 * p.npml for n in p.shape]
    ncell = n2[0] * n2[1] * n2[2]
    slab = sum(2 * p.npml * (ncell // n2[a]) for a in range(3))
    return int(ncell * (8 * s + 2 * m) + slab * 4 * psi)


def eiso_bytes_per_step(p, nshots, s, m=4, split=None):
    """shots (N_int 10 s + N_pml 20 p) + N_all 3 m, p the split parts' width
    (= s, or 4 for block storage, whose split parts stay FP32)."""
    split = s if split is None else split
    nall = p.cells
    nint = p.nx * p.nz
    return int(nshots * (nint * 10 * s + (nall - nint) * 20 * split) + nall * 3 * m)


def ecyl_bytes_per_step(p, s, m=4):
    """cells (9 fields read and written, 8 materials read) + the CPML memory
    variables of the z strips (6) and the outer radial strip (12 for mode 0,
    18 for n > 0), each read and written."""
    npml = p.np_used
    nx2, nz2 = p.nx + npml, p.nz + 2 * npml
    nr = 18 if p.n > 0 else 12
    return nx2 * nz2 * (18 * s + 8 * m) + 2 * s * (6 * nx2 * 2 * npml + nr * npml * nz2)


def make_workload(name, size=None):
    from seismod_b200 import workloads as W
    if name == "ecyl":
        p = W.ecyl_case(nx=2000, nz=4000, npml=20, nsteps=1000, n=1, src="Fz", nrec=64, seed=7)
        return ("ecyl", p, "e_cyl_iso 2000 x 4000 (r x z, +20 CPML), dr = dz = 1 m, azimuthal "
                           "mode 1, Fz source, 1000-step shot")
    if name == "a3d" and size:
        return ("a3d", W.cfg1(n=size),
                f"a_iso_3d {size}^3 (+2x16 CPML), dx 5 m, cfg1 model family, 1000-step shot")
    if name == "a3d":
        return "a3d", W.cfg1(), "a_iso_3d 256^3 (+2x16 CPML = 288^3), dx 5 m, 1000-step shot"
    if name == "a3d512":
        return "a3d", W.cfg3(), "a_iso_3d 512^3 (+2x16 CPML = 544^3), dx 5 m, 2000-step shot"
    if name == "eiso":
        return ("eiso", W.cfg2(),
                "e_iso 1000x500 (+2x20 PML), 64 shots batched, 2000-step shots")
    if name == "eiso1":
        return "eiso", W.cfg0(), "e_iso 400x400 (+2x20 PML), single shot, 1500-step shot"
    if name in ("serve", "serve_overload"):
        # 1.25 arrivals/s is about 0.8 x the capacity the request loop showed
        # under overload (1.6 shots/s at 4 arrivals/s) on this mix
        rate = 1.25 if name == "serve" else 4.0
        return ("serve", W.cfg4(rate_hz=rate),
                f"request stream: 64 Poisson arrivals at {rate:g}/s, 70% e_iso 200^2..2000^2, "
                "30% a_iso_3d 128^3..384^3, 500..3000 steps, seeded layered models")
    raise SystemExit(f"unknown workload {name}")


# ----------------------------------------------------------------------------
# our arm
# ----------------------------------------------------------------------------

# DRAM bytes (read + written) per step of the dominant kernel(s), measured
# with ncu on B200 for exactly these workloads (profiles/ holds the
# summaries and the commands): the interior + ring launches of a_iso_3d
# 288^3 in FP32 and block storage (224^3 captures scaled by the cell count,
# which traffic follows), e_iso 64 x 1040 x 540 in FP32 and block storage,
# and the velocity + stress launches of e_cyl_iso 2020 x 4040 FP32.
MEASURED_TRAFFIC = {
    ("a3d", 256, "fp32"): 1.125e9,
    ("a3d", 256, "bfp16"): 0.809e9,
    ("eiso", 1000, "fp32"): 1.8166e9,
    ("eiso", 1000, "bfp16"): 1.1759e9,
    ("ecyl", 2000, "fp32"): 1.1106e9,
}


def measured_traffic(kind, p, prec):
    edge = p.shape[0] if kind == "a3d" else p.nx
    return MEASURED_TRAFFIC.get((kind, edge, prec))


def max_over_ranks(x, dist, device):
    """The largest x over all ranks: the job's time is its slowest rank's.
    dist is torch.distributed (initialised, any backend) or None."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_gcells(cells, K, world, ms):
    """Whole-job throughput of replicas: every rank updates `cells` cells per
    step for K steps; ms is the slowest rank's time."""
    return cells * K * world / (ms * 1e-3) / 1e9


def trace_err(a, b):
    a = np.concatenate([np.ravel(x) for x in a])
    b = np.concatenate([np.ravel(x) for x in b])
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


TUNE = True
GRAPH = 16
LAUNCH = {}   # (workload kind, precision) -> the autotuner's launch configuration


def device_for(kind, p, precision, dev_id, shots=None):
    from seismod_b200 import api
    if kind == "ecyl":
        return api.ecyl_device(p, precision, dev_id)   # one launch shape, no graphs
    if kind == "a3d":
        dev, n = api.a3d_device(p, precision, dev_id)
    else:
        dev, n = api.eiso_device(p, precision, shots, dev_id)
    if GRAPH:
        dev.set_graph(GRAPH)   # before the tuning, so its trials run as the steps will
    if TUNE:
        LAUNCH[(kind, precision)] = dev.autotune()[:-1]
    return dev, n


def time_steps(dev, K, torch):
    ext = torch.cuda.ExternalStream(dev.stream())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    dev.sync()
    e0.record(ext)
    dev.run(K)
    e1.record(ext)
    e1.synchronize()
    return e0.elapsed_time(e1)


def run_ours(args, rank, world, local_rank, torch, dist):
    from seismod_b200 import api
    kind, p, desc = make_workload(args.workload, args.size)
    prec = args.precision
    sbytes = {"fp32": 4, "fp64": 8, "fp16": 2, "bf16": 2,
              "bfp16": A3D_BFP_BYTES if kind == "a3d" else EISO_BFP_BYTES}[prec]
    mbytes = 8 if prec == "fp64" else 4
    nshots = len(p.shots) if kind == "eiso" else 1
    if kind == "a3d":
        bps = a3d_bytes_per_step(p, sbytes, mbytes, 4 if prec == "bfp16" else None)
        cells = p.cells
    elif kind == "ecyl":
        bps = ecyl_bytes_per_step(p, sbytes, mbytes)
        cells = p.cells
    else:
        bps = eiso_bytes_per_step(p, nshots, sbytes, mbytes)
        cells = p.cells * nshots
    dev, nsteps_shot = device_for(kind, p, prec, local_rank)
    K, Wm = args.steps, args.warmup
    dev.run(Wm)
    # one more untimed graph's worth of steps: the time loop's CUDA graph is
    # captured here (a one-off cost of the handle, like the autotuning)
    if GRAPH and kind != "ecyl":
        dev.run(GRAPH)
    dev.sync()
    dev.kernel_stats(reset=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with Clocks(local_rank) as clk:
        ms = time_steps(dev, K, torch)
    _, _, launches = dev.kernel_stats(reset=True)
    ms = max_over_ranks(ms, dist, f"cuda:{local_rank}")
    # dominant-kernel duration: separate pass with per-launch events (event
    # nodes inside the graph replays when the handle replays graphs)
    dev.set_timing(True)
    Kr = max(100, min(K, 400))   # at least 100 launches: the mean of a short pass is noisy
    if GRAPH and kind != "ecyl":
        Kr = -(-Kr // GRAPH) * GRAPH   # whole graphs only
    dev.run(Kr)
    upd_ms, upd_n, _ = dev.kernel_stats(reset=True)
    dev.set_timing(False)
    dev.close()
    value = job_gcells(cells, K, world, ms)
    hbm, how = peaks()
    achieved = bps / (upd_ms / upd_n * 1e-3) / 1e9
    out = {
        "metric": METRIC, "value": round(value, 3), "unit": "Gcell/s",
        "n_gpus": world, "steps": K, "warmup": Wm, "ms_per_step": round(ms / K, 5),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if prec == "fp64" else "f32",
        "data": "synthetic (seeded generator of the named configuration; no dataset exists)",
        "config": {"workload": desc, "precision": f"{prec} storage",
                   "cells_per_shot": p.cells, "shots": nshots * world,
                   "parallelism": f"replicas x{world} (shot-parallel, no collective)",
                   "l2": "inputs larger than L2 (state %.0f MB)" % (bps / 1e6),
                   "launch": {"autotuned": TUNE, "config_chunk": LAUNCH.get((kind, prec)),
                              "graph_steps": GRAPH if kind != "ecyl" else 0,
                              "untimed_graph_capture_steps": GRAPH if kind != "ecyl" else 0}},
        "shots_per_s": round(nshots * world / (ms / K * 1e-3 * nsteps_shot), 3),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm,
                     "unit": "GB/s", "frac": round(achieved / hbm, 4),
                     "traffic": measured_traffic(kind, p, prec),
                     "peak_source": how, "algorithmic_bytes_per_step": bps,
                     "duration": "mean of %d update launches, CUDA events on the library's "
                                 "stream%s, right after the timed region"
                                 % (upd_n, " recorded as event nodes of the replayed graphs"
                                    if GRAPH and kind != "ecyl" else ""),
                     "kernel": "wavefield update (velocity + stress/pressure, PML/CPML)"},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    return out, kind, p, desc, cells


def precision_side(kind, p, local_rank, K):
    """Throughput of the other storage precisions and every trace error
    against an FP64 device run of the whole shot."""
    from seismod_b200 import api
    import torch
    run = api.run_a3d if kind == "a3d" else (lambda q, pr, d: api.run_eiso(q, pr, [0], d)[0])
    if kind == "ecyl":
        run = api.run_ecyl
    precs = ("fp32",) if kind == "ecyl" else ("fp32", "bfp16", "fp16", "bf16")
    res = {}
    # the rates first (warm-up and graph capture untimed), then the long
    # whole-shot runs for the trace errors
    for prec in precs:
        try:
            dev, _ = device_for(kind, p, prec, local_rank)
            dev.run(10 + (GRAPH if kind != "ecyl" else 0))
            ms = time_steps(dev, 200, torch)
            dev.close()
            res[prec] = {"ms_per_step": round(ms / 200, 5)}
        except Exception as e:  # report, do not hide
            res[prec] = {"error": str(e)[:200]}
    ref64 = run(p, "fp64", local_rank)
    for prec in precs:
        if "error" in res[prec]:
            continue
        try:
            res[prec] = {"trace_err_vs_fp64": trace_err(run(p, prec, local_rank), ref64),
                         **res[prec]}
        except Exception as e:  # report, do not hide
            res[prec] = {"error": str(e)[:200]}
    return res


def timed_rate(kind, p, prec, dev_id, steps, shots=None):
    """(ms per step of the whole step, mean step-kernel ms per step) of an
    autotuned, graph-replayed handle: 5 warm-up steps, then `steps` steps
    timed with CUDA events on the handle's stream, then the same number with
    per-launch events around the step kernel."""
    import torch
    dev, _ = device_for(kind, p, prec, dev_id, shots)
    dev.run(5 + GRAPH)   # warm-up, and the time loop's CUDA graph captured
    dev.sync()
    ms = time_steps(dev, steps, torch) / steps
    dev.set_timing(True)
    dev.run(-(-steps // GRAPH) * GRAPH if GRAPH and kind != "ecyl" else steps)
    kms, kn, _ = dev.kernel_stats(reset=True)
    dev.set_timing(False)
    dev.close()
    return ms, kms / max(kn, 1)


def headline(local_rank, cfg1_precisions):
    """The metric's comparison, measured in the default run: the plain
    single-shot FP32 form against the batched forms (64 shots of the 1040 x
    540 e_iso model in one handle, FP32 and 16-bit block storage) in shots/s,
    each form's trace error against an FP64 run of the same shot, and the
    roofline fraction of the batched step kernels; the a_iso_3d shots in FP32
    and block storage (256^3 from the main run, 512^3 here); the 400 x 400
    e_iso shot.  Step counts are fixed (not --steps) so every entry is a
    stable rate; whole shots (2000 / 1500 steps) give the trace errors."""
    from seismod_b200 import api
    from seismod_b200 import workloads as W
    hbm, how = peaks()
    out = {"peak_gbs": hbm, "peak_source": how}
    # ---- e_iso 1000 x 500 (+2x20 PML), 64 shots, 2000 steps ----
    p = W.cfg2()
    n = api.nsteps(p.duration, p.dt)
    nsh = len(p.shots)
    # every rate before the long whole-shot runs (reference and trace errors),
    # each on a GPU in the same state
    ms1, _ = timed_rate("eiso", p, "fp32", local_rank, 400, shots=[0])
    rates = {prec: timed_rate("eiso", p, prec, local_rank, 200) for prec in ("fp32", "bfp16")}
    ref = {s: api.run_eiso(p, "fp64", [s], local_rank)[0] for s in (0, nsh - 1)}
    e = {}
    err1 = trace_err(api.run_eiso(p, "fp32", [0], local_rank)[0], ref[0])
    sps1 = 1.0 / (ms1 * 1e-3 * n)
    e["single_shot_fp32"] = {"ms_per_step": round(ms1, 5), "shots_per_s": round(sps1, 3),
                             "trace_err_vs_fp64": err1,
                             "l2": "state of one shot fits in L2 (no flush): favours this "
                                   "baseline, so the batched ratios are lower bounds"}
    for prec in ("fp32", "bfp16"):
        ms, kms = rates[prec]
        batch = api.run_eiso(p, prec, None, local_rank)
        err = max(trace_err(batch[s], ref[s]) for s in ref)
        bps = eiso_bytes_per_step(p, nsh, EISO_BFP_BYTES if prec == "bfp16" else 4.0, 4,
                                  4.0 if prec == "bfp16" else None)
        sps = nsh / (ms * 1e-3 * n)
        e[f"batched_{prec}"] = {
            "ms_per_step": round(ms, 5), "shots_per_s": round(sps, 3),
            "speedup_vs_single_fp32": round(sps / sps1, 3), "trace_err_vs_fp64": err,
            "kernel_ms_per_step": round(kms, 5), "algorithmic_bytes_per_step": bps,
            "roofline_frac": round(bps / (kms * 1e-3) / 1e9 / hbm, 4),
            "l2": "inputs larger than L2"}
    out["eiso_1040x540_64shots"] = e
    b = e["batched_bfp16"]
    out["batched_bfp16_vs_single_fp32"] = {
        "shots_per_s_ratio": b["speedup_vs_single_fp32"],
        "trace_err_vs_fp64": b["trace_err_vs_fp64"],
        "meets_2x_at_1e-3": bool(b["speedup_vs_single_fp32"] >= 2.0 and b["trace_err_vs_fp64"] <= 1e-3)}
    # ---- a_iso_3d 256^3 (the main run's shot) ----
    if cfg1_precisions:
        out["a3d_288cube"] = {k: cfg1_precisions[k] for k in ("fp32", "bfp16") if k in cfg1_precisions}
    # ---- a_iso_3d 512^3 (+2x16 CPML = 544^3), 2000 steps ----
    q = W.cfg3()
    # rates first: right after the long FP64 reference shot the GPU runs hot
    # (a 100-step FP32 rate taken there read 1.6-2.0 ms against 1.3)
    rates = {prec: timed_rate("a3d", q, prec, local_rank, 100) for prec in ("fp32", "bfp16")}
    ref3 = api.run_a3d(q, "fp64", local_rank)
    a = {}
    for prec in ("fp32", "bfp16"):
        ms, kms = rates[prec]
        err = trace_err(api.run_a3d(q, prec, local_rank), ref3)
        sb = A3D_BFP_BYTES if prec == "bfp16" else 4.0
        bps = a3d_bytes_per_step(q, sb, 4, 4 if prec == "bfp16" else None)
        a[prec] = {"ms_per_step": round(ms, 5), "gcell_per_s": round(q.cells / (ms * 1e-3) / 1e9, 3),
                   "shots_per_s": round(1.0 / (ms * 1e-3 * 2000), 4),
                   "trace_err_vs_fp64": err, "kernel_ms_per_step": round(kms, 5),
                   "algorithmic_bytes_per_step": bps,
                   "roofline_frac": round(bps / (kms * 1e-3) / 1e9 / hbm, 4),
                   "l2": "inputs larger than L2"}
    out["a3d_544cube_2000steps"] = a
    del q, ref3
    # ---- e_iso 400 x 400 (+2x20 PML), one shot, 1500 steps ----
    c0 = W.cfg0()
    ms0, _ = timed_rate("eiso", c0, "fp32", local_rank, 1500)
    out["eiso_440sq_single_fp32"] = {
        "ms_per_step": round(ms0, 5), "gcell_per_s": round(c0.cells / (ms0 * 1e-3) / 1e9, 3),
        "l2": "state fits in L2 (launch-bound shot; no flush)"}
    return out


def batching_side(p, local_rank, K, batched_ms):
    """Shots/s of the plain single-shot FP32 form (one shot per handle) against
    the batched forms, and each form's trace error against an FP64 run of the
    same shot."""
    from seismod_b200 import api
    import torch
    nsh = len(p.shots)
    n = api.nsteps(p.duration, p.dt)
    ref64 = api.run_eiso(p, "fp64", [0], local_rank)[0]
    out = {}
    dev, _ = device_for("eiso", p, "fp32", local_rank, shots=[0])
    dev.run(10)
    k1 = min(K, 400)
    ms1 = time_steps(dev, k1, torch) / k1
    dev.close()
    tr = api.run_eiso(p, "fp32", [0], local_rank)[0]
    out["single_shot_fp32"] = {"ms_per_step": round(ms1, 5),
                               "shots_per_s": round(1.0 / (ms1 * 1e-3 * n), 3),
                               "trace_err_vs_fp64": trace_err(tr, ref64)}
    for prec in ("fp32", "fp16", "bf16"):
        if prec == "fp32" and batched_ms is not None:
            ms = batched_ms
        else:
            dev, _ = device_for("eiso", p, prec, local_rank)
            dev.run(10)
            kb = min(K, 200)
            ms = time_steps(dev, kb, torch) / kb
            dev.close()
        tr = api.run_eiso(p, prec, [0], local_rank)[0]
        sps = nsh / (ms * 1e-3 * n)
        out[f"batched_{prec}"] = {"ms_per_step": round(ms, 5), "shots_per_s": round(sps, 3),
                                  "speedup_vs_single_fp32": round(sps * ms1 * 1e-3 * n, 3),
                                  "trace_err_vs_fp64": trace_err(tr, ref64)}
    return out


def run_serve(args, local_rank):
    """The mixed request stream through the request loop: each request is
    built on the host and submitted at its arrival time; value = cell updates
    of completed requests / (first submit -> last completion)."""
    from seismod_b200 import serving
    _, reqs, desc = make_workload(args.workload)
    srv = serving.Server(device=local_rank, max_active=16, slice_steps=64,
                         graph_steps=GRAPH or 0, group=args.group)
    t0 = time.perf_counter()
    lag = []
    with Clocks(local_rank) as clk:
        for r in reqs:
            now = time.perf_counter() - t0
            if r.arrival > now:
                time.sleep(r.arrival - now)
            lag.append(max(0.0, time.perf_counter() - t0 - r.arrival))
            srv.submit(r.kind, r.problem, args.precision)
        srv.drain()
    st = srv.stats()
    srv.close()
    out = {
        "metric": METRIC, "value": round(st["gcell_per_s"], 3), "unit": "Gcell/s",
        "n_gpus": 1, "steps": len(reqs), "warmup": 0,
        "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32",
        "data": "synthetic (seeded request stream of the named configuration)",
        "config": {"workload": desc, "precision": f"{args.precision} storage",
                   "server": "max_active 16, slices of 64 steps, CUDA graphs of %d steps%s"
                             % (GRAPH or 0, ", e_iso and a_iso_3d requests each stepped as "
                                "one group" if args.group else "")},
        "serving": {"shots_per_s": round(st["shots_per_s"], 4),
                    "latency_p50_s": round(st["latency_p50"], 4),
                    "latency_p99_s": round(st["latency_p99"], 4),
                    "wait_p50_s": round(st["wait_p50"], 4), "wait_p99_s": round(st["wait_p99"], 4),
                    "completed": st["completed"], "failed": st["failed"],
                    "busy_s": round(st["busy_s"], 3), "max_running": st["max_running"],
                    "hbm_peak_gb": round(st["hbm_peak"] / 1e9, 2),
                    "hbm_budget_gb": round(st["hbm_budget"] / 1e9, 2),
                    "submit_lag_p99_s": round(float(np.percentile(lag, 99)), 3)},
        "clocks": clk.summary(),
    }
    return out


def e2e(kind, p, K, local_rank):
    """Whole user call through the public API from host arrays: set-up and
    upload, K steps, traces back to the host, teardown."""
    from seismod_b200 import api
    import gc
    gc.collect()   # the earlier legs' garbage is not this call's to collect
    marks = [("start", time.perf_counter())]
    if kind == "a3d":   # the steps of api.a3d_device, timed one by one
        q = api.a3d_inputs(p, pad=False)   # padded as it is staged
        marks.append(("host_inputs", time.perf_counter()))
        dev = api.A3DDevice(q["vp"], q["rho"], q["npml"], q["d"], q["dt"], q["coef"], "fp32",
                            local_rank, padded=False)
        dev.set_sources(*q["src"], q["src_scale"])
        dev.set_receivers(*q["rec"], q["nsteps"])
        marks.append(("create_upload", time.perf_counter()))
        if TUNE:
            dev.autotune()
        if GRAPH:
            dev.set_graph(GRAPH)
        marks.append(("tune_graph", time.perf_counter()))
    else:
        dev, _ = device_for(kind, p, "fp32", local_rank)
        marks.append(("setup", time.perf_counter()))
    dev.run(K)
    dev.sync()
    marks.append(("steps", time.perf_counter()))
    if kind == "a3d":
        tr = dev.traces_array()
        d2h = tr.size * 8
    elif kind == "ecyl":
        tr = dev.traces()
        d2h = sum(len(x) for x in tr) * 8
    else:
        tr = [dev.traces_array(s) for s in range(dev.nshots)]
        d2h = sum(t.size for t in tr) * 8
    marks.append(("traces_back", time.perf_counter()))
    dev.close()
    marks.append(("teardown", time.perf_counter()))
    wall = marks[-1][1] - marks[0][1]
    phases = {marks[k][0]: round(marks[k][1] - marks[k - 1][1], 4) for k in range(1, len(marks))}
    if kind == "a3d":
        n2 = [n + 2 * p.npml for n in p.shape]
        pitch = math.ceil(n2[2] / 32) * 32
        h2d = 2 * n2[0] * n2[1] * pitch * 4
        cells = p.cells
    elif kind == "ecyl":
        pitch = math.ceil((p.nz + 2 * p.np_used) / 32) * 32
        h2d = 8 * (p.nx + p.np_used) * pitch * 4   # the eight materials
        cells = p.cells
    else:
        pitch = math.ceil((p.nz + 2 * p.npml) / 32) * 32
        h2d = 5 * (p.nx + 2 * p.npml) * pitch * 4
        cells = p.cells * len(p.shots)
    return {"value": round(cells * K / wall / 1e9, 3), "unit": "Gcell/s",
            "h2d_bytes_per_step": int(h2d / K), "d2h_bytes_per_step": int(d2h / K),
            "wall_s": round(wall, 3), "phases_s": phases}


# ----------------------------------------------------------------------------
# the reference on the host cores
# ----------------------------------------------------------------------------

def _raise_nofile():
    soft, hard = resource.getrlimit(resource.RLIMIT_NOFILE)
    try:
        resource.setrlimit(resource.RLIMIT_NOFILE, (hard, hard))
    except Exception:
        pass
    return resource.getrlimit(resource.RLIMIT_NOFILE)[0]


def reference_rate(kind, p, steps):
    """Gcell/s of the reference program over `steps` steps of p (time of a
    (2 + steps)-step run minus a 2-step run, same inputs).  The model is
    written as a 1-D profile file (the reference's own shortcut) so parsing
    stays short; the arithmetic per step does not depend on the values."""
    from oracle import oracle as O
    from seismod_b200 import workloads as W
    if not O.ref_available():
        return None, "reference build absent (oracle/_ref)"
    nofile = _raise_nofile()
    d = tempfile.mkdtemp(prefix="refbench_")
    q = p
    nrec = len(p.receivers)
    if nrec + 64 > nofile:  # the reference keeps one open file per trace
        q = dataclasses.replace(p, receivers=p.receivers[: max(nofile - 64, 1)])
    prog = "a_iso_3d" if kind == "a3d" else ("e_iso" if p.nx <= p.nz else "e_iso_lrfix")
    if kind == "ecyl":
        prog = "e_cyl_iso"
    pars = []
    for n in (2, 2 + steps):
        r = dataclasses.replace(q, duration=W.steps_duration(n, q.dt_ms))
        if kind in ("a3d", "ecyl"):
            pars.append(r.write(os.path.join(d, f"n{n}"), profile_1d=True))
        else:
            pars.append(r.write(os.path.join(d, f"n{n}"), shot=0, profile_1d=True))
    # each length twice, the faster run of each kept: start-up (model read,
    # allocation) varies from run to run and would otherwise leak into the
    # difference
    times = [min(O.run_reference(prog, par, os.path.dirname(par), timeout=3600)
                 for _ in range(2)) for par in pars]
    dt = (times[1] - times[0]) / steps
    how = f"time(2+{steps} steps) - time(2 steps), fastest of two runs each"
    if dt <= 0:   # start-up noise larger than the steps: bound by the whole run
        dt = times[1] / (2 + steps)
        how = f"time(2+{steps} steps) / {2 + steps} (start-up included: the difference was not positive)"
    cells = p.cells
    threads = 4 if kind == "ecyl" else 3
    sample = (f"{prog} (oracle/_ref, gcc -O3, OpenMP, {threads} threads as hard-coded), "
              f"{steps} steps of the full grid, {len(q.receivers)} receivers, "
              f"1-D profile model file; {how}")
    return cells / dt / 1e9, sample


def run_reference_arm(args, rank, world):
    if rank != 0:
        return None
    kind, p, desc = make_workload(args.workload)
    if kind == "serve":
        # the reference serves nothing: one program per shot; its rate on the
        # stream's first e_iso request stands for the stream
        p = next(r.problem for r in p if r.kind == "eiso")
        kind = "eiso"
    # a fixed sample per workload (not --steps: a few steps would leave the
    # timing to start-up noise), a few tens of seconds of host time at most
    steps = 12 if kind == "a3d" else (20 if kind == "ecyl" else 200)
    rate, sample = reference_rate(kind, p, steps)
    if rate is None:
        return {"impl": "reference", "unavailable": sample}
    return {"impl": "reference", "metric": METRIC, "value": round(rate, 4), "unit": "Gcell/s",
            "n_gpus": world, "steps": steps, "warmup": args.warmup,
            "ms_per_step": round(p.cells / (rate * 1e9) * 1e3, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": desc},
            "cpu_baseline": {"value": round(rate, 4), "unit": "Gcell/s",
                             "cores": 4 if kind == "ecyl" else 3,
                             "kind": "reference", "sample": sample},
            "e2e": {"value": round(rate, 4), "unit": "Gcell/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


# ----------------------------------------------------------------------------

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="a3d",
                    choices=["a3d", "a3d512", "eiso", "eiso1", "ecyl", "serve", "serve_overload"])
    ap.add_argument("--precision", default="fp32",
                    choices=["fp32", "fp64", "fp16", "bf16", "bfp16"])
    ap.add_argument("--no-side", action="store_true", help="skip precision / CPU side runs")
    ap.add_argument("--no-headline", action="store_true",
                    help="skip the batched / 512^3 / 400^2 comparison of the default run")
    ap.add_argument("--no-tune", action="store_true", help="default launch configuration")
    ap.add_argument("--group", action="store_true",
                    help="serve workloads: running requests of one program take their slices "
                         "together (one launch per step over all their grids)")
    ap.add_argument("--no-graph", action="store_true", help="launch every kernel from the host")
    ap.add_argument("--size", type=int, default=None,
                    help="a3d only: interior edge length instead of 256 (profiling captures)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    global TUNE, GRAPH
    TUNE = not args.no_tune
    GRAPH = 0 if args.no_graph else 16

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        out = run_reference_arm(args, rank, world)
        if out is not None:
            print(json.dumps(out), flush=True)
        return 0

    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    if args.workload in ("serve", "serve_overload"):
        if rank == 0:
            print(json.dumps(run_serve(args, local_rank)), flush=True)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return 0
    out, kind, p, desc, cells = run_ours(args, rank, world, local_rank, torch, dist)
    if rank == 0 and not args.no_side and kind == "eiso" and len(p.shots) > 1:
        out["batching"] = batching_side(p, local_rank, args.steps, out["ms_per_step"])
    if rank == 0 and not args.no_side:
        out["precisions"] = precision_side(kind, p, local_rank, args.steps)
        if args.workload == "a3d" and args.size is None and not args.no_headline:
            try:
                out["headline"] = headline(local_rank, out["precisions"])
            except Exception as e:  # report, do not hide
                out["headline"] = {"error": str(e)[:300]}
        out["e2e"] = e2e(kind, p, args.steps, local_rank)
        steps = 12 if kind == "a3d" else (20 if kind == "ecyl" else 200)
        rate, sample = reference_rate(kind, p, steps)
        if rate is not None:
            out["cpu_baseline"] = {"value": round(rate, 4), "unit": "Gcell/s",
                                   "cores": 4 if kind == "ecyl" else 3,
                                   "kind": "reference", "sample": sample}
        else:
            out["cpu_baseline"] = {"value": None, "unit": "Gcell/s", "cores": 0,
                                   "kind": "reference", "sample": sample}
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
