#!/usr/bin/env python3
"""Benchmark: k-tensors/hour and GLUPS of the B200 permeability solver.

Workload (one bench step = one full permeability tensor): the 128^3 packing
of overlapping prolate ellipsoids, semi-axes (4, 4, 12) voxels along z,
porosity 0.45, percolating in x, y and z (seeded, synthetic), solved along
+x, +y and +z with g = 1e-6 (--ff 4), tau = 1, eps = 1e-6 relative drift every
1000 steps, hold 2, min 4000, max 50000 steps, 2000 averaging steps.  The
three directions run concurrently on one GPU.

Reported (one JSON line, rank 0):
  value      k-tensors/hour of the headline path, the fastest of FP32
             populations, FP16 populations and the tau = 1 FP32 moment forms that
             stays within 1e-3 of the FP64 tensor (every path keeps the
             reference's stopping rule), inputs resident in HBM, device time
             from CUDA events on the solver's stream;
  e2e        the same through the public API with the structure in host memory
             (host->device copy and result read-back inside the timed region);
  plain_fp32 the same workload with plain FP32 storage, one launch per step;
  serving    p50/p99 latency of a short 20 requests/s Poisson trace through the
             continuous-batching server;
  rel_err    the headline K against the FP64 K of the same structure;
  roofline   HBM roofline of the step kernel: algorithmic bytes (pore voxels
             x 2 x 19 x element size + N/8 mask) / time, against the measured
             copy bandwidth;
  cpu_baseline  the reference CPU solver (oracle/_ref/lbm3d-perm, built from
             the reference sources) on all host cores, a bounded fixed-step
             sample, extrapolated to a converged tensor with the FP64 step
             counts.

Multi-GPU (torchrun): every rank solves its own tensors, no collective in the
data path ("weak" scaling); the timed region is bracketed by a barrier and the
max over ranks is reported.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp16]
    python bench.py --impl reference        # the reference CPU solver alone
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "k-tensors/hr & GLUPS at ≤1e-3 rel err vs FP64, vs plain FP32; p50/p99 latency"
WORKLOAD = dict(workload="perm-tensor 128^3 prolate-ellipsoid packing (4,4,12) phi=0.45, 3 directions",
                n=128, semi=(4.0, 4.0, 12.0), porosity=0.45, seed=0, ff=4.0, tau=1.0, eps=1e-6,
                lag=1000, hold=2, min_steps=4000, max_steps=50000, avg_steps=2000)
# algorithmic bytes per pore-voxel update: populations read + written once
# (AA pattern), or for the tau = 1 moment form a 20-byte record read + written
BYTES_PER_UPDATE = {"fp64": 304, "fp32": 152, "fp16": 76, "bf16": 76, "m32": 40, "m64": 80}


def alg_bytes_per_dir_step(prec, npore, nvox):
    """Algorithmic DRAM bytes of one direction-step: pore-voxel state read and
    written once plus the bit mask; the dense moment form (md32) reads a
    20-byte record and a mask byte for every voxel of the box and writes the
    pore voxels' records."""
    if prec == "md32":
        return 20.0 * nvox + 20.0 * npore + 1.0 * nvox
    return npore * BYTES_PER_UPDATE[prec] + nvox / 8.0


DTYPE = {"fp16": "f16-storage/f32-compute/f64-reduce", "bf16": "bf16-storage/f32-compute/f64-reduce",
         "fp32": "f32-storage/f32-compute/f64-reduce", "fp64": "f64",
         "m32": "f32 moment records (tau=1)/f32-compute/f64-reduce", "m64": "f64 moment records (tau=1)",
         "md32": "f32 dense moment records (tau=1)/f32-compute/f64-reduce"}
# Steps per direction of the converged FP64 solve of the workload structure
# (x, y, z).  Our FP64 path reproduces the reference's step counts exactly
# (per-step bit-identical populations; see tests/test_gpu_solve3d.py); the
# reference arm uses these to turn its fixed-step sample into a full tensor.
FP64_STEPS = (8000, 7000, 8000)



def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ----------------------------------------------------------------- clocks --
class Clocks:
    """nvidia-smi sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,clocks.mem")

    def __init__(self, device):
        self.device = device
        self.p = None

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            self.f = tempfile.TemporaryFile(mode="w+")
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                       "-lms", "200", "-i", str(self.device)], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        return self

    def __exit__(self, *exc):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(5)
            except Exception:
                self.p.kill()

    def summary(self):
        if not self.p:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.f.seek(0)
        sm, smax, mem, watts, reasons = [], [], [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.f:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
                watts.append(float(parts[3]))
                if len(parts) > 9:
                    mem.append(float(parts[9]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "mem_mhz": statistics.median(mem) if mem else None,
                "power_w": statistics.median(watts) if watts else None,
                "samples": len(sm), "reasons": sorted(reasons)}


# ----------------------------------------------------------------- helpers --
def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def profiled_traffic(prec):
    """DRAM bytes (read + write) per step launch of a path's step kernels, the
    mean of one odd and one even launch, from the committed ncu summary."""
    for p in sorted((ROOT / "profiles").glob("*_tensor128.md")):
        m = re.search(r"traffic_bytes_per_launch\[" + re.escape(prec) + r"\]:\s*([0-9.eE+]+)", p.read_text())
        if m:
            return float(m.group(1))
    return None


def tensor_K(runs, mu, F):
    return np.array([[mu * runs[j].q[c] / F for j in range(3)] for c in range(3)])


def k_errors(K, K64):
    """Per-entry relative error of K against the FP64 K; off-diagonals are
    judged against the trace scale (they are ~0 for this axis-aligned packing)."""
    scale = np.abs(np.diag(K64)).max()
    diag = float(max(abs(K[i, i] - K64[i, i]) / abs(K64[i, i]) for i in range(3)))
    off = float(max(abs(K[i, j] - K64[i, j]) for i in range(3) for j in range(3) if i != j) / scale)
    return {"max_rel_diag": diag, "max_offdiag_over_kmax": off, "max_rel": max(diag, off)}


class EventTimer:
    """CUDA events on the solver's stream (every kernel of the context runs there)."""

    def __init__(self, torch, stream_ptr):
        self.torch = torch
        self.stream = torch.cuda.ExternalStream(stream_ptr)

    def __enter__(self):
        self.e0 = self.torch.cuda.Event(enable_timing=True)
        self.e1 = self.torch.cuda.Event(enable_timing=True)
        self.torch.cuda.synchronize()
        self.e0.record(self.stream)
        return self

    def __exit__(self, *exc):
        self.e1.record(self.stream)
        self.e1.synchronize()
        self.torch.cuda.synchronize()
        self.ms = self.e0.elapsed_time(self.e1)


# ------------------------------------------------------------ CPU baseline --
def cpu_sample(solid, wl, seconds_target=12.0, steps=None):
    """Reference binary (or the oracle port) on all host cores, fixed-step sample.

    Returns dict(lups_per_core, cores, kind, sample, seconds)."""
    from oracle import oracle as O
    from flow_anizotropy_b200.structure_io3d import save_structure
    cores = os.cpu_count() or 1
    nz, ny, nx = solid.shape
    N = solid.size
    ref = O.ref_binary("lbm3d-perm")
    if steps is None:
        steps = max(2, int(seconds_target * 12e6 / (3 * N)))       # ~12 MLUPS per core
    tmp = Path(tempfile.mkdtemp(prefix="lbmcpu_"))
    raw = tmp / "s.raw"
    save_structure(raw, solid)
    t0 = time.perf_counter()
    if ref is not None:
        kind = "reference"
        args = ["--quiet", "--ff", str(wl["ff"]), "--max-steps", str(steps), "--min-steps", str(steps + 1),
                "--lag", str(steps + 1), "--avg-steps", "0"]
        procs = [subprocess.Popen([str(ref), str(raw), str(tmp / f"o{i}.csv")] + args,
                                  stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL) for i in range(cores)]
        for p in procs:
            p.wait()
        dirs = 3
    else:
        kind = "port"
        cores = 1
        st = O.State3D(solid, wl["tau"])
        st.reset([2.5e-7 * wl["ff"], 0, 0])
        st.step(steps)
        dirs = 1
    dt = time.perf_counter() - t0
    shutil.rmtree(tmp, ignore_errors=True)
    lups = dirs * steps * N / dt          # all-node convention, per process
    return dict(lups_per_core=lups, cores=cores, kind=kind, seconds=dt,
                sample=f"{dirs} x {steps} fixed steps of the {nx}x{ny}x{nz} workload structure per process, "
                       f"{cores} processes")


def cpu_baseline_entry(cpu, N, steps64):
    """k-tensors/hour of the CPU solver extrapolated with the FP64 step counts."""
    lu_tensor = N * float(sum(steps64))
    sec_tensor = lu_tensor / cpu["lups_per_core"]
    return {"value": 3600.0 * cpu["cores"] / sec_tensor, "unit": "k-tensors/hr", "cores": cpu["cores"],
            "kind": cpu["kind"], "sample": cpu["sample"] + "; extrapolated with FP64 step counts "
            f"{list(map(int, steps64))}", "mlups_per_core": cpu["lups_per_core"] / 1e6}


# ---------------------------------------------------------------- serving ----
def serve_trace(device, prec, args):
    """Short Poisson trace at the serving rate (20 requests/s) through the
    continuous-batching server: structures of the uneven-size mix restricted
    to its two smallest edges (48, 64) so the trace drains in seconds."""
    from flow_anizotropy_b200 import structures as st
    from flow_anizotropy_b200.serve import Server, poisson_arrivals, replay
    from flow_anizotropy_b200.solver import Params3D
    mix = [d for d in st.batch_mix(64, seed=5) if d["n"] in (48, 64)][:8]
    pool = [st.make(d) for d in mix]
    F = 2.5e-7 * WORKLOAD["ff"]
    p = Params3D(tau=1.0, eps=WORKLOAD["eps"], lag=WORKLOAD["lag"], hold=WORKLOAD["hold"],
                 min_steps=WORKLOAD["min_steps"], max_steps=WORKLOAD["max_steps"],
                 avg_steps=WORKLOAD["avg_steps"], precision=prec)
    forces = [[F, 0, 0], [0, F, 0], [0, 0, F]]
    srv = Server(precision=prec, hbm_budget=150 * 2**30, chunk=128, device=device, variant=args.serve_variant)
    arrivals = poisson_arrivals(20.0, args.serve_seconds, seed=11)
    t0 = time.perf_counter()
    stats = replay(srv, arrivals, lambda i: (pool[i % len(pool)], forces, p))
    wall = time.perf_counter() - t0
    srv.close()
    served = stats.completed / wall
    # plain FP32 on the same structures, one tensor at a time, each with the
    # step-kernel variant the autotuner picks for it (tuning not timed): the
    # baseline the served throughput is compared with
    from flow_anizotropy_b200 import solver as S
    tuned = [S.tune3d(s_, ndir=3, precision="fp32", nsteps=100, device=device)[0] for s_ in pool]
    pps = [Params3D(**{**p.__dict__, "precision": "fp32", "variant": v}) for v in tuned]
    S.solve3d(pool[0], forces, pps[0], device=device)
    t0 = time.perf_counter()
    for s_, pp in zip(pool, pps):
        S.solve3d(s_, forces, pp, device=device)
    plain = len(pool) / (time.perf_counter() - t0)
    return {"rate_per_s": 20.0, "arrival_seconds": args.serve_seconds, "requests": stats.completed,
            "p50_s": stats.pct(50), "p99_s": stats.pct(99), "max_resident": stats.max_resident,
            "p50_queue_s": float(np.percentile(stats.queue_waits, 50)) if stats.queue_waits else None,
            "k_tensors_per_hr": 3600.0 * served, "served_per_s": served, "overloaded": 20.0 > served,
            "plain_fp32_per_s": plain, "speedup_vs_plain_fp32": served / plain,
            "admission": f"FIFO, HBM budget 150 GiB, resident work cap {srv.max_work} pore-voxel-directions",
            "mix": "batch mix, edges 48 and 64 only (8 seeded structures, reused)", "path": prec,
            "batch_variant": args.serve_variant}


# -------------------------------------------------------------- our arm ----
def run_ours(args, rank, world, local_rank):
    import torch
    from flow_anizotropy_b200 import _lib
    from flow_anizotropy_b200 import solver as S
    from flow_anizotropy_b200 import structures as st

    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    device = local_rank
    torch.cuda.set_device(device)
    wl = dict(WORKLOAD)
    solid = st.ellipsoid_packing(wl["n"], wl["semi"], wl["porosity"], wl["seed"])
    N = solid.size
    npore = int((solid == 0).sum())
    F = 2.5e-7 * wl["ff"]
    forces = [[F, 0, 0], [0, F, 0], [0, 0, F]]
    mu = (1.0 / 3.0) * (wl["tau"] - 0.5)
    ctx = _lib.context(device)
    solid_dev = torch.from_numpy(np.ascontiguousarray(solid)).cuda(device)

    def params(prec, variant=0):
        return S.Params3D(tau=wl["tau"], eps=wl["eps"], lag=wl["lag"], hold=wl["hold"], min_steps=wl["min_steps"],
                          max_steps=wl["max_steps"], avg_steps=wl["avg_steps"], precision=prec,
                          criterion="auto", variant=variant)

    # FP64 oracle solve on the GPU (the reference's arithmetic), untimed
    r64, _, _ = S.solve3d(solid_dev, forces, params("fp64"), device=device)
    K64 = tensor_K(r64, mu, F)
    steps64 = [r.steps for r in r64]

    def measure(prec, warmup, steps, host_input=False):
        best, ms = S.tune3d(solid, ndir=3, precision=prec, nsteps=100, device=device)
        p = params(prec, best)
        inp = solid if host_input else solid_dev
        for _ in range(warmup):
            S.solve3d(inp, forces, p, device=device)
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        runs_all = []
        torch.cuda.nvtx.range_push(f"timed:{prec}{':e2e' if host_input else ''}")
        with Clocks(device) as clk, EventTimer(torch, ctx.stream) as t:
            for _ in range(steps):
                runs, rc, _ = S.solve3d(inp, forces, p, device=device)
                runs_all.append(runs)
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        ms_total = t.ms
        if dist is not None:
            tt = torch.tensor([ms_total], dtype=torch.float64, device=f"cuda:{device}")
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            ms_total = float(tt.item())
        dir_steps = sum(sum(r.steps for r in runs) for runs in runs_all)
        launches = sum(max(r.steps for r in runs) for runs in runs_all)
        return dict(prec=prec, variant=best, tune_ms=ms, ms=ms_total, runs=runs_all[-1], clocks=clk.summary(),
                    dir_steps=dir_steps, launches=launches)

    results = {}
    cands = [args.precision] if args.precision != "auto" else ["fp32", "fp16", "m32", "md32"]
    if "fp32" not in cands:
        cands.append("fp32")
    for prec in cands:
        m = measure(prec, args.warmup, args.steps)
        m["K"] = tensor_K(m["runs"], mu, F)
        m["err"] = k_errors(m["K"], K64)
        results[prec] = m

    def rates(m):
        sec = m["ms"] / 1e3
        tensors = world * args.steps
        return (3600.0 * tensors / sec, world * m["dir_steps"] * npore / sec / 1e9,
                world * m["dir_steps"] * N / sec / 1e9)

    ok = [p_ for p_ in results if results[p_]["err"]["max_rel"] <= 1e-3]
    head_prec = max(ok, key=lambda p_: rates(results[p_])[0]) if ok else "fp32"
    head = results[head_prec]
    plain = results["fp32"]
    e2e = measure(head_prec, 1, args.steps, host_input=True)
    kt, gf, ga = rates(head)
    kt_p, gf_p, ga_p = rates(plain)
    kt_e, _, _ = rates(e2e)
    peak, peak_kind = measured_peak()
    alg_bytes = head["dir_steps"] * alg_bytes_per_dir_step(head_prec, npore, N)
    achieved = alg_bytes / (head["ms"] / 1e3) / 1e9
    per_launch_alg = alg_bytes / max(1, head["launches"])
    traffic = profiled_traffic(head_prec)
    serving = serve_trace(device, args.serve_precision, args) if args.serve_seconds > 0 else None
    out = None
    if rank == 0:
        cpu = cpu_sample(solid, wl, seconds_target=args.cpu_seconds)
        cpu_entry = cpu_baseline_entry(cpu, N, steps64)
        paths = {}
        for p_, m in results.items():
            k_, g_, a_ = rates(m)
            paths[p_] = {"k_tensors_per_hr": k_, "glups_fluid": g_, "glups_all_node": a_,
                         "steps_per_direction": [r.steps for r in m["runs"]],
                         "converged": [r.converged for r in m["runs"]],
                         "rel_err_vs_fp64": m["err"], "kernel_variant": m["variant"],
                         "hbm_gbs_alg": m["dir_steps"] * alg_bytes_per_dir_step(p_, npore, N) / (m["ms"] / 1e3) / 1e9,
                         "clocks": m["clocks"]}
        out = {
            "metric": METRIC, "value": kt, "unit": "k-tensors/hr", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": head["ms"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": DTYPE[head_prec],
            "data": "synthetic (seeded structure; no dataset)",
            "config": {"workload": wl["workload"], "seed": wl["seed"], "tau": wl["tau"], "g": F,
                       "eps": wl["eps"], "lag": wl["lag"], "hold": wl["hold"], "min_steps": wl["min_steps"],
                       "max_steps": wl["max_steps"], "avg_steps": wl["avg_steps"],
                       "path": head_prec, "kernel_variant": head["variant"],
                       "criterion": "block means, batch-means SE, k-sigma" if head_prec in ("fp16", "bf16") else "drift (reference)",
                       "parallelism": f"work partition x{world} (one tensor stream per GPU)",
                       "l2": "lattices (3 x 19 x 0.94 M pores x elem: 215 MB fp32, 108 MB fp16) stream from HBM "
                             "every step; inputs are the whole tensor solve, not a cached kernel"},
            "glups_fluid": gf, "glups_all_node": ga,
            "steps_per_direction": [r.steps for r in head["runs"]],
            "rel_err_vs_fp64": head["err"],
            "paths": paths,
            "plain_fp32": {"value": kt_p, "unit": "k-tensors/hr", "glups_fluid": gf_p, "glups_all_node": ga_p},
            "speedup_vs_plain_fp32": kt / kt_p,
            "fp64_steps_per_direction": steps64,
            "serving": serving,
            "e2e": {"value": kt_e, "unit": "k-tensors/hr", "h2d_bytes_per_step": int(N),
                    "d2h_bytes_per_step": int(3 * 64)},
            "gpu_launches": int(head["launches"] + 8 * args.steps),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": traffic, "alg_bytes_per_launch": per_launch_alg,
                         "kernel": f"step3d ({head_prec}) variant {head['variant']}"},
            "cpu_baseline": cpu_entry,
            "clocks": head["clocks"],
        }
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return out


# ------------------------------------------------------- batched workload --
def _make_structure(d):
    from flow_anizotropy_b200 import structures as st
    return st.make(d)


def run_batch_workload(args, device=0):
    """The uneven-size mix: `count` structures with edges from {48,64,96,128,160},
    three directions each, solved (a) one structure at a time with plain FP32
    per-step launches, (b) all resident in one batch (CUDA-graph chunks,
    per-solve retirement) for each batched path.  Reports k-tensors/hour."""
    import multiprocessing as mproc
    import torch
    from flow_anizotropy_b200 import _lib
    from flow_anizotropy_b200 import solver as S
    from flow_anizotropy_b200 import structures as st
    mix = st.batch_mix(args.count, seed=0)
    with mproc.get_context("spawn").Pool(min(16, os.cpu_count() or 1)) as pool:
        structs = pool.map(_make_structure, mix)
    F = 2.5e-7 * WORKLOAD["ff"]
    forces = [[F, 0, 0], [0, F, 0], [0, 0, F]]
    ctx = _lib.context(device)

    def params(prec):
        return S.Params3D(tau=1.0, eps=WORKLOAD["eps"], lag=WORKLOAD["lag"], hold=WORKLOAD["hold"],
                          min_steps=WORKLOAD["min_steps"], max_steps=WORKLOAD["max_steps"],
                          avg_steps=WORKLOAD["avg_steps"], precision=prec)

    out = {"workload": f"batch mix of {args.count} structures (edges 48..160, 3 directions)",
           "voxels": int(sum(s.size for s in structs)), "pores": int(sum((s == 0).sum() for s in structs))}
    ref = {}
    with EventTimer(torch, ctx.stream) as t:
        for i, s_ in enumerate(structs):
            runs, _, _ = S.solve3d(s_, forces, params("fp32"), device=device)
            ref[i] = runs
    out["plain_fp32_per_solve"] = {"seconds": t.ms / 1e3, "k_tensors_per_hr": 3600 * len(structs) / (t.ms / 1e3)}
    for prec in args.batch_paths.split(","):
        b = S.Batch(precision=prec, hbm_budget=150 * 2**30, chunk=256, device=device)
        done = {}
        with EventTimer(torch, ctx.stream) as t:
            for i, s_ in enumerate(structs):
                assert b.submit(s_, forces, params(prec), tag=i)
            while len(done) < len(structs):
                b.run(4)
                done.update(dict(b.poll()))
        b.close()
        worst = 0.0
        for i in done:
            for a_, m_ in zip(ref[i], done[i]):
                sc = np.abs(a_.q).max()
                worst = max(worst, float(np.abs(a_.q - m_.q).max() / sc))
        out[f"batched_{prec}"] = {"seconds": t.ms / 1e3, "k_tensors_per_hr": 3600 * len(structs) / (t.ms / 1e3),
                                  "max_rel_q_vs_plain_fp32": worst}
    out["speedup_vs_plain_fp32"] = {k: out["plain_fp32_per_solve"]["seconds"] / v["seconds"]
                                    for k, v in out.items() if k.startswith("batched_")}
    return out


def run_large_workload(args, device=0):
    """The large configuration: 512^3 Gaussian random field (sigma (3, 3, 9),
    phi = 0.15, largest cluster spanning z), tau = 0.8, three directions
    resident; a fixed number of steps (--large-steps) per storage precision,
    timed with CUDA events after the autotuner's pick: fluid GLUPS and the
    HBM roofline of the step kernels (a converged tensor at this size takes
    tens of thousands of steps, beyond a bench run)."""
    import torch
    from flow_anizotropy_b200 import _lib
    from flow_anizotropy_b200 import solver as S
    from flow_anizotropy_b200 import structures as st
    solid = st.large_grf(0, n=args.large_n)
    npore, N = int((solid == 0).sum()), solid.size
    dev = torch.from_numpy(np.ascontiguousarray(solid)).cuda(device)
    ctx = _lib.context(device)
    F = 1e-6
    forces = [[F, 0, 0], [0, F, 0], [0, 0, F]]
    peak, peak_kind = measured_peak()
    out = {"workload": f"{args.large_n}^3 GRF sigma (3,3,9) phi=0.15 largest z-spanning cluster, tau 0.8, 3 directions",
           "pore_voxels": npore, "voxels": N, "steps": args.large_steps, "paths": {}}
    for prec in ("fp32", "fp16"):
        best, _ = S.tune3d(solid, ndir=3, precision=prec, nsteps=50, device=device)
        p = S.Params3D(tau=0.8, eps=0.0, lag=10**9, hold=10**6, min_steps=0, max_steps=args.large_steps,
                       avg_steps=0, precision=prec, criterion="drift", variant=best)
        S.solve3d(dev, forces, S.Params3D(**{**p.__dict__, "max_steps": 20}), device=device)
        with Clocks(device) as clk, EventTimer(torch, ctx.stream) as t:
            runs, _, _ = S.solve3d(dev, forces, p, device=device)
        upd = 3.0 * npore * args.large_steps
        ab = 3.0 * args.large_steps * alg_bytes_per_dir_step(prec, npore, N)
        out["paths"][prec] = {"ms": t.ms, "glups_fluid": upd / (t.ms / 1e3) / 1e9, "kernel_variant": best,
                              "roofline": {"achieved": ab / (t.ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                                           "frac": ab / (t.ms / 1e3) / 1e9 / peak, "peak_kind": peak_kind},
                              "clocks": clk.summary()}
    return out


def run_gen_workload(args, device=0):
    """Structure generation (the gen_aniso_structures3d.py dataset model,
    default knobs) at --gen-size: samples/s of the device generator against
    the CPU restatement of the reference's per-voxel work (numpy field and
    quantile, scipy labelling of the 3x3x3 tiling) on one host core, on the
    same samples; the structures are checked to be identical."""
    import torch
    from flow_anizotropy_b200 import _lib
    from flow_anizotropy_b200 import gen3d as G
    from oracle import gen3d_oracle as GO
    n = args.count
    gen = G.Generator(size=args.gen_size)
    gen.sample(0)                                        # warm-up
    ctx = _lib.context(device)
    with EventTimer(torch, ctx.stream) as t:
        t0 = time.perf_counter()
        got = [gen.sample(i) for i in range(1, n + 1)]
        wall = time.perf_counter() - t0
    attempts = sum(r[1]["attempts"] for r in got if r is not None)
    cpu_n = max(1, min(n, 3))
    t0 = time.perf_counter()
    ref = [GO.sample(i, args.gen_size) for i in range(1, cpu_n + 1)]
    cpu = time.perf_counter() - t0
    same = all(np.array_equal(a[0], b[0]) for a, b in zip(got[:cpu_n], ref) if a is not None and b is not None)
    return {"workload": f"gen_aniso_structures3d model, {args.gen_size}^3, default knobs, {n} samples",
            "samples_per_s": n / wall, "attempts": attempts, "device_ms": t.ms,
            "cpu_baseline": {"samples_per_s": cpu_n / cpu, "cores": 1, "kind": "port",
                             "sample": f"{cpu_n} samples, numpy field + quantile, scipy labelling"},
            "speedup_vs_cpu_core": (n / wall) / (cpu_n / cpu), "identical_structures": same}


def run_perm2d_workload(args, device=0):
    """D2Q9 permeability (the 2D drop-in's solve) of --count seeded 256^2
    disc packings (solid fraction 0.2-0.4), forcing along x and y, the 2D
    reference's default convergence knobs, --group2d images per launch
    (lbm_solve2d_many): images/s, fluid GLUPS and the HBM roofline (72 B per
    fluid-cell update) against the reference binary lbm2d-perm on all host
    cores (fixed-step sample per process, extrapolated with the device step
    counts, which equal the reference's: the 2D path is bit-identical)."""
    import torch
    from oracle import oracle as O
    from flow_anizotropy_b200 import _lib
    from flow_anizotropy_b200 import solver as S
    from flow_anizotropy_b200 import structures as st
    from flow_anizotropy_b200.structure_io import save_dat
    n, group = args.count, args.group2d
    imgs = np.stack([st.disc_packing_2d(seed=i, solid_fraction=0.2 + 0.05 * (i % 5)) for i in range(n)])
    F = S.FX_BASE
    forces = [[F, 0.0], [0.0, F]]
    p = S.Params2D()
    ctx = _lib.context(device)
    S.solve2d_many(imgs[:min(group, n)], forces, S.Params2D(max_steps=200, min_steps=100, lag=100, avg_steps=0),
                   device=device)
    runs = []
    with Clocks(device) as clk, EventTimer(torch, ctx.stream) as t:
        t0 = time.perf_counter()
        for g in range(0, n, group):
            runs += S.solve2d_many(imgs[g:g + group], forces, p, device=device)[0]
        wall = time.perf_counter() - t0
    steps = [r.steps for rr in runs for r in rr]
    fluid = float((imgs == 0).sum(axis=(1, 2)).mean())
    upd = sum(r.steps * float((img == 0).sum()) for img, rr in zip(imgs, runs) for r in rr)
    peak, peak_kind = measured_peak()
    ab = 72.0 * upd
    out = {"workload": f"D2Q9 256^2 disc packings, {n} images x 2 directions, reference 2D defaults "
                       f"(eps 1e-3, lag 5000, min 10000, avg 20000), {group} images per launch",
           "images_per_s": n / (t.ms / 1e3), "images_per_s_wall": n / wall, "device_ms": t.ms,
           "glups_fluid": upd / (t.ms / 1e3) / 1e9, "mean_fluid_cells": fluid,
           "steps_min_max": [min(steps), max(steps)], "converged": sum(r.converged for rr in runs for r in rr),
           "roofline": {"bound": "hbm", "achieved": ab / (t.ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                        "frac": ab / (t.ms / 1e3) / 1e9 / peak, "peak_kind": peak_kind},
           "clocks": clk.summary()}
    ref = O.ref_binary("lbm2d-perm")
    if ref is not None:
        cores = os.cpu_count() or 1
        sample_steps = max(2, int(args.cpu_seconds * 20e6 / (2 * 65536)))   # ~20 MLUPS per core
        tmp = Path(tempfile.mkdtemp(prefix="lbm2dcpu_"))
        save_dat(tmp / "s.dat", imgs[0])
        argv = ["--quiet", "--max-steps", str(sample_steps), "--min-steps", str(sample_steps + 1),
                "--lag", str(sample_steps + 1), "--avg-steps", "0", "--avg-sample", "1"]
        t0 = time.perf_counter()
        procs = [subprocess.Popen([str(ref), str(tmp / "s.dat"), str(tmp / f"o{i}.csv")] + argv,
                                  stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL) for i in range(cores)]
        for pr in procs:
            pr.wait()
        dt = time.perf_counter() - t0
        shutil.rmtree(tmp, ignore_errors=True)
        lups = 2 * sample_steps * 65536 / dt          # per process, all cells
        sec_image = sum(steps) / n * 65536 / lups     # both directions of a mean image
        out["cpu_baseline"] = {"images_per_s": cores / sec_image, "cores": cores, "kind": "reference",
                               "mlups_per_core": lups / 1e6,
                               "sample": f"2 x {sample_steps} fixed steps of a 256^2 image per process, "
                                         f"{cores} processes; extrapolated with the device step counts"}
        out["speedup_vs_cpu"] = out["images_per_s"] / out["cpu_baseline"]["images_per_s"]
    return out


# -------------------------------------------------------- reference arm ----
def run_reference(args, rank, world):
    if rank != 0:
        return None
    from flow_anizotropy_b200 import structures as st
    wl = dict(WORKLOAD)
    solid = st.ellipsoid_packing(wl["n"], wl["semi"], wl["porosity"], wl["seed"])
    N = solid.size
    steps64 = FP64_STEPS
    per_step = []
    cpu = None
    for i in range(args.warmup + args.steps):
        cpu = cpu_sample(solid, wl, seconds_target=args.cpu_seconds)
        if i >= args.warmup:
            per_step.append(cpu)
    lups = statistics.median(c["lups_per_core"] for c in per_step)
    cpu = dict(per_step[-1], lups_per_core=lups)
    entry = cpu_baseline_entry(cpu, N, steps64)
    return {"metric": METRIC, "value": entry["value"], "unit": "k-tensors/hr", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * float(sum(steps64)) * N / (lups * cpu["cores"]), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded structure)",
            "config": {"workload": wl["workload"], "seed": wl["seed"], "precision": "fp64"},
            "impl": "reference", "cpu_baseline": entry,
            "e2e": {"value": entry["value"], "unit": "k-tensors/hr", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="auto", choices=["auto", "fp16", "bf16", "fp32", "fp64", "m32", "md32"])
    ap.add_argument("--serve-seconds", type=float, default=5.0)
    ap.add_argument("--serve-precision", default="fp16", choices=["fp32", "fp16", "bf16"])
    ap.add_argument("--serve-variant", type=int, default=1,
                    help="step-kernel variant of the serving batch (-1: library default; 1 measured "
                         "fastest for FP16 on the 48^3-64^3 serving mix)")
    ap.add_argument("--workload", default="tensor128", choices=["tensor128", "batch", "gen3d", "large", "perm2d"])
    ap.add_argument("--group2d", type=int, default=16, help="images per launch of the perm2d workload")
    ap.add_argument("--large-n", type=int, default=512, help="cell edge of the large workload")
    ap.add_argument("--large-steps", type=int, default=2000)
    ap.add_argument("--gen-size", type=int, default=80, help="cell edge of the gen3d workload")
    ap.add_argument("--count", type=int, default=32, help="structures of the batch workload")
    ap.add_argument("--batch-paths", default="fp32,m32,fp16")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        out = run_reference(args, rank, world)
    elif args.workload == "batch":
        out = run_batch_workload(args, local_rank) if rank == 0 else None
    elif args.workload == "gen3d":
        out = run_gen_workload(args, local_rank) if rank == 0 else None
    elif args.workload == "large":
        out = run_large_workload(args, local_rank) if rank == 0 else None
    elif args.workload == "perm2d":
        out = run_perm2d_workload(args, local_rank) if rank == 0 else None
    else:
        out = run_ours(args, rank, world, local_rank)
    if out is not None and rank == 0:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
