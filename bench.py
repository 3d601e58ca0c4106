#!/usr/bin/env python3
"""Benchmark: k-tensors/hour and GLUPS of the B200 permeability solver.

Workload (one bench step = one full permeability tensor): the 128^3 packing
of overlapping prolate ellipsoids, semi-axes (4, 4, 12) voxels along z,
porosity 0.45, percolating in x, y and z (seeded, synthetic), solved along
+x, +y and +z with g = 1e-6 (--ff 4), tau = 1, eps = 1e-6, every 1000 steps,
hold 2, min 4000, max 50000 steps, 2000 averaging steps.  The three
directions run concurrently on one GPU.

Stopping rules: FP64 and FP32 storage stop by the reference's rule (relative
drift of q between checks, LMB3d/lbm3d-perm.cpp:332-364); FP16 and BF16
storage stop by a block-mean test (the 2D reference's k-sigma test,
LMB2d/main.cpp:123-178, with batch-means standard errors), because their
stochastic rounding keeps q wandering at the 1e-6 level the drift test uses.
Every path's tensor is compared with the FP64 tensor and with the row the
reference binary wrote for this structure (tests/golden/configs/).

Reported (one JSON line, rank 0):
  value      k-tensors/hour of the headline path: the fastest of FP32, FP16
             and BF16 storage whose every k_ij is within 1e-3 of FP64; inputs
             resident in HBM, device time from CUDA events on the solver's
             stream;
  e2e        the same through the public API with the structure in host memory
             (host->device copy and result read-back inside the timed region);
  paths      every storage path: k-tensors/h, GLUPS, the 3x3 per-k_ij error
             matrix against FP64 and against the reference row;
  mean_velocity  superficial q (the reference's output) and the pore mean
             q / phi of each forcing direction;
  serving    the continuous-batching server on the serving mix (batch-mix
             structures, one 256^3 GRF in every 20 requests) at 20 requests/s
             for --serve-seconds, p50/p99 latency of what completed (that rate
             overloads one GPU, so these latencies are mostly queueing), and
             `sustained`: the same mix at --serve-sustained of the rate served,
             every request run to completion, p50/p99 of all of them;
  large      512^3 GRF, tau 0.8, fixed steps: GLUPS and roofline per path;
  perm2d     the D2Q9 solver (the 2D drop-in's solve) on --perm2d-images
             seeded 256^2 disc packings with the 2D reference's defaults:
             images/s, GLUPS, roofline, the reference binary on the host cores;
  plain64    the 64^3 FP64 single-solve configuration: time per tensor, q_x,
             q_x / phi, k_xx, step counts and K against the reference
             binary's row, and the reference binary on the host cores;
  batch      a sample of the 256-structure uneven-size mix, batched against
             one structure at a time in plain FP32;
  roofline   HBM roofline of the step kernels: algorithmic bytes (pore voxels
             x 2 x 19 x element size + N/8 mask) / time, against the measured
             copy bandwidth;
  cpu_baseline  the reference CPU solver (oracle/_ref/lbm3d-perm, built from
             the reference sources) on all host cores, a bounded fixed-step
             sample, extrapolated to a converged tensor with the step counts
             the reference itself took on this structure.

Multi-GPU (torchrun): every rank solves its own tensors, no collective in the
data path ("weak" scaling); the timed region is bracketed by a barrier and the
max over ranks is reported.  The serving, large and batch legs run at N = 1.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp16]
    python bench.py --impl reference        # the reference CPU solver alone
    python bench.py --workload steps --precision fp16 --variant V --steps 12   # profiling runs
"""
from __future__ import annotations

import argparse
import json
import math
import os
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
TAGS = ("fx", "fy", "fz")
# Row the reference binary appended for the workload structure
# (tests/golden/make_golden_configs.py); its step counts turn the CPU sample
# into a converged tensor, and its tensor is the reference every path is
# compared with.
REF_ROW = ROOT / "tests" / "golden" / "configs" / "precision128.csv"


def reference_row(path=REF_ROW):
    """Steps, fluxes and K of the reference's row, or None if it is absent."""
    if not Path(path).exists():
        return None
    lines = Path(path).read_text().splitlines()
    row = dict(zip(lines[0].split(","), lines[1].split(",")))
    meta = json.loads(Path(path).with_suffix(".json").read_text())
    return {"steps": [int(row[f"steps_{t}"]) for t in TAGS],
            "q": np.array([[float(row[f"q{c}_{t}"]) for c in "xyz"] for t in TAGS]),
            "K": np.array([[float(row[f"K_{a}{b}"]) for b in "xyz"] for a in "xyz"]),
            "sha256": meta["sha256"], "seconds": meta["seconds"], "path": str(Path(path).relative_to(ROOT))}


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


TRAFFIC = ROOT / "profiles" / "traffic.json"


def profiled_traffic(prec, variant, updates_per_launch):
    """DRAM bytes (read + write) per step launch of this run's step kernels,
    from the ncu captures recorded in profiles/traffic.json (per precision, a
    list of kernel variants, each per pore-voxel update: the mean of one odd
    and one even launch, with the command that measured it), scaled to this
    run's updates per launch.  None when no capture of this precision and
    kernel variant is recorded."""
    if not TRAFFIC.exists():
        return None
    recs = json.loads(TRAFFIC.read_text()).get(prec) or []
    if isinstance(recs, dict):
        recs = [recs]
    for rec in recs:
        if rec.get("variant") == variant:
            return rec["dram_bytes_per_update"] * updates_per_launch
    return None


def tensor_K(runs, mu, F):
    return np.array([[mu * runs[j].q[c] / F for j in range(3)] for c in range(3)])


def k_errors(K, Kref):
    """Per-entry error of K against Kref: |dK_ij| / |Kref_ij| on the diagonal,
    / max_i |Kref_ii| off it (the off-diagonals of this axis-aligned packing
    are differences of nearly cancelling sums, ~1e-3 of the diagonal)."""
    scale = np.abs(np.diag(Kref)).max()
    den = np.where(np.eye(3, dtype=bool), np.abs(Kref), scale)
    m = np.abs(K - Kref) / den
    diag = float(np.diag(m).max())
    off = float(m[~np.eye(3, dtype=bool)].max())
    return {"matrix": m.tolist(), "max_rel_diag": diag, "max_offdiag_over_kmax": off,
            "max_rel": max(diag, off)}


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


def cpu_baseline_entry(cpu, N, steps, steps_source):
    """k-tensors/hour of the CPU solver: its measured all-node rate on the
    fixed-step sample, extrapolated to a converged tensor with `steps`."""
    lu_tensor = N * float(sum(steps))
    sec_tensor = lu_tensor / cpu["lups_per_core"]
    return {"value": 3600.0 * cpu["cores"] / sec_tensor, "unit": "k-tensors/hr", "cores": cpu["cores"],
            "kind": cpu["kind"], "extrapolated": True,
            "formula": "cores x 3600 / (N x sum(steps) / all-node LUPS per core)",
            "steps_per_tensor": list(map(int, steps)), "steps_source": steps_source,
            "sample": cpu["sample"], "sample_seconds": cpu["seconds"],
            "mlups_per_core": cpu["lups_per_core"] / 1e6}


# ---------------------------------------------------------------- serving ----
def _serve_pool_entry(d):
    from flow_anizotropy_b200 import structures as st
    return st.make(d)


def serve_trace(device, prec, args):
    """The serving configuration: a Poisson stream at 20 requests/s for
    --serve-seconds; every request is a structure of the uneven-size batch
    mix (edges 48..160), and every 20th a 256^3 Gaussian-random-field sample
    (phi in U[0.15, 0.35]), each asking for a 3-direction tensor at eps 1e-6
    under a 150 GiB admission budget.  The requests draw from a pool of
    seeded structures built before the trace (structure generation is not
    timed).  At this rate the GPU is overloaded, so the trace runs for the
    arrival window and stops: throughput is the requests completed in the
    window, latencies are those of the completed requests, and the queue left
    at the end is reported.  The plain FP32 rate is the same mix solved one
    structure at a time."""
    import multiprocessing as mproc
    from flow_anizotropy_b200 import solver as S
    from flow_anizotropy_b200 import structures as st
    from flow_anizotropy_b200.serve import Server, poisson_arrivals, replay
    descs = [st.serving_request(i, seed=3) for i in range(args.serve_pool * 20 // 19 + 40)]
    mix_d = [d for d in descs if d["kind"] != "grf"][:args.serve_pool]
    grf_d = [d for d in descs if d["kind"] == "grf"][:2]
    with mproc.get_context("spawn").Pool(min(16, os.cpu_count() or 1)) as pool:
        built = pool.map(_serve_pool_entry, mix_d + grf_d)
    mix, grf = built[:len(mix_d)], built[len(mix_d):]
    F = 2.5e-7 * WORKLOAD["ff"]
    p = S.Params3D(tau=1.0, eps=WORKLOAD["eps"], lag=WORKLOAD["lag"], hold=WORKLOAD["hold"],
                   min_steps=WORKLOAD["min_steps"], max_steps=WORKLOAD["max_steps"],
                   avg_steps=WORKLOAD["avg_steps"], precision=prec)
    forces = [[F, 0, 0], [0, F, 0], [0, 0, F]]

    def request(i):
        if i % 20 == 19:
            return grf[(i // 20) % len(grf)], forces, p
        return mix[(i - i // 20) % len(mix)], forces, p

    srv = Server(precision=prec, hbm_budget=150 * 2**30, chunk=128, device=device, variant=args.serve_variant)
    arrivals = poisson_arrivals(20.0, args.serve_seconds, seed=11)
    t0 = time.perf_counter()
    stats = replay(srv, arrivals, request, horizon=args.serve_seconds)
    wall = time.perf_counter() - t0
    queued, resident = len(srv.queue), len(srv.inflight)
    srv.close()
    served = stats.completed / wall
    # the same mix at a load the GPU sustains (a fraction of the rate just
    # served): every request runs to completion, so p50/p99 are the solver's
    # latency under continuous batching rather than the overloaded queue's
    sus = None
    if args.serve_sustained > 0 and served > 0:
        rate2 = args.serve_sustained * served
        srv2 = Server(precision=prec, hbm_budget=150 * 2**30, chunk=128, device=device, variant=args.serve_variant)
        arr2 = poisson_arrivals(rate2, args.serve_seconds, seed=12)
        t0 = time.perf_counter()
        st2 = replay(srv2, arr2, request)
        wall2 = time.perf_counter() - t0
        srv2.close()
        lat2 = np.array(st2.latencies) if st2.latencies else np.array([np.nan])
        sus = {"rate_per_s": rate2, "load_fraction": args.serve_sustained, "arrival_seconds": args.serve_seconds,
               "arrived": len(arr2), "completed": st2.completed, "wall_seconds": wall2,
               "p50_s": float(np.percentile(lat2, 50)), "p99_s": float(np.percentile(lat2, 99)),
               "p50_queue_s": float(np.percentile(st2.queue_waits, 50)) if st2.queue_waits else None,
               "max_resident": st2.max_resident, "k_tensors_per_hr": 3600.0 * st2.completed / wall2}
    # plain FP32, one structure at a time with the library's default FP32
    # kernels, on a sample of the same mix weighted as the stream is (19 mix
    # requests to 1 GRF)
    pp = S.Params3D(**{**p.__dict__, "precision": "fp32"})
    nplain = min(len(mix), args.serve_plain_sample)
    S.solve3d(mix[0], forces, pp, device=device)
    t0 = time.perf_counter()
    for s_ in mix[:nplain]:
        S.solve3d(s_, forces, pp, device=device)
    t_mix = (time.perf_counter() - t0) / nplain
    t0 = time.perf_counter()
    S.solve3d(grf[0], forces, pp, device=device)
    t_grf = time.perf_counter() - t0
    plain = 1.0 / (0.95 * t_mix + 0.05 * t_grf)
    lat = np.array(stats.latencies) if stats.latencies else np.array([np.nan])
    return {"rate_per_s": 20.0, "arrival_seconds": args.serve_seconds, "arrived": len(arrivals),
            "completed": stats.completed, "left_queued": queued, "left_resident": resident,
            "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "p50_queue_s": float(np.percentile(stats.queue_waits, 50)) if stats.queue_waits else None,
            "k_tensors_per_hr": 3600.0 * served, "served_per_s": served, "overloaded": 20.0 > served,
            "max_resident": stats.max_resident, "max_resident_gib": stats.max_resident_bytes / 2**30,
            "plain_fp32_per_s": plain,
            "plain_fp32_sample": f"{nplain} mix structures + 1 GRF, weighted 19:1",
            "speedup_vs_plain_fp32": served / plain,
            "admission": f"FIFO, HBM budget 150 GiB, resident work cap {srv.max_work} pore-voxel-directions",
            "mix": f"pool of {len(mix)} batch-mix structures (edges {sorted(set(d['n'] for d in mix_d))}) "
                   f"and {len(grf)} 256^3 GRF samples (every 20th request)",
            "path": prec, "batch_variant": args.serve_variant,
            "latency_note": "latencies of the requests completed within the window (an overloaded "
                            "server's queue grows without bound, so they understate the steady state)",
            "sustained": sus}


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
    phi = npore / N
    F = 2.5e-7 * wl["ff"]
    forces = [[F, 0, 0], [0, F, 0], [0, 0, F]]
    mu = (1.0 / 3.0) * (wl["tau"] - 0.5)
    ctx = _lib.context(device)
    solid_dev = torch.from_numpy(np.ascontiguousarray(solid)).cuda(device)
    ref = reference_row()
    if ref is not None:
        import hashlib
        if hashlib.sha256(np.ascontiguousarray(solid).tobytes()).hexdigest() != ref["sha256"]:
            log("reference row was written for another structure: not used")
            ref = None

    def params(prec, variant=0):
        return S.Params3D(tau=wl["tau"], eps=wl["eps"], lag=wl["lag"], hold=wl["hold"], min_steps=wl["min_steps"],
                          max_steps=wl["max_steps"], avg_steps=wl["avg_steps"], precision=prec,
                          criterion="auto", variant=variant)

    # FP64 solve on the GPU (the reference's arithmetic), untimed
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
    cands = [args.precision] if args.precision != "auto" else ["fp32", "fp16", "bf16"]
    if "fp32" not in cands:
        cands.append("fp32")
    for prec in cands:
        m = measure(prec, args.warmup, args.steps)
        m["K"] = tensor_K(m["runs"], mu, F)
        m["err"] = k_errors(m["K"], K64)
        m["err_ref"] = k_errors(m["K"], ref["K"]) if ref is not None else None
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
    updates_per_launch = head["dir_steps"] * npore / max(1, head["launches"])
    traffic = profiled_traffic(head_prec, head["variant"], updates_per_launch)
    legs = world == 1
    serving = serve_trace(device, args.serve_precision, args) if legs and args.serve_seconds > 0 else None
    large = run_large_workload(args, device) if legs and args.large_steps > 0 else None
    plain64 = run_plain64_leg(args, device) if legs and args.plain64_reps > 0 and rank == 0 else None
    batch = run_batch_workload(args, device) if legs and args.count > 0 else None
    perm2d = None
    if legs and args.perm2d_images > 0 and rank == 0:
        a2 = argparse.Namespace(**{**vars(args), "count": args.perm2d_images,
                                   "cpu_seconds": min(args.cpu_seconds, 6.0)})
        perm2d = run_perm2d_workload(a2, device)
    out = None
    if rank == 0:
        cpu = cpu_sample(solid, wl, seconds_target=args.cpu_seconds)
        if ref is not None:
            cpu_entry = cpu_baseline_entry(cpu, N, ref["steps"], f"the reference's own run ({ref['path']})")
        else:
            cpu_entry = cpu_baseline_entry(cpu, N, steps64, "the GPU FP64 solve (no reference row present)")
        paths = {}
        for p_, m in results.items():
            k_, g_, a_ = rates(m)
            paths[p_] = {"k_tensors_per_hr": k_, "glups_fluid": g_, "glups_all_node": a_,
                         "steps_per_direction": [r.steps for r in m["runs"]],
                         "converged": [r.converged for r in m["runs"]],
                         "rel_err_vs_fp64": m["err"], "rel_err_vs_reference": m["err_ref"],
                         "kernel_variant": m["variant"],
                         "hbm_gbs_alg": m["dir_steps"] * alg_bytes_per_dir_step(p_, npore, N) / (m["ms"] / 1e3) / 1e9,
                         "clocks": m["clocks"]}
        qh = np.array([r.q for r in head["runs"]])
        out = {
            "metric": METRIC, "value": kt, "unit": "k-tensors/hr", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": head["ms"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": DTYPE[head_prec],
            "data": "synthetic (seeded structure; no dataset)",
            "config": {"workload": wl["workload"], "seed": wl["seed"], "tau": wl["tau"], "g": F,
                       "eps": wl["eps"], "lag": wl["lag"], "hold": wl["hold"], "min_steps": wl["min_steps"],
                       "max_steps": wl["max_steps"], "avg_steps": wl["avg_steps"],
                       "path": head_prec, "kernel_variant": head["variant"],
                       "criterion": "block means, batch-means SE, k-sigma" if head_prec in ("fp16", "bf16")
                       else "drift (reference)",
                       "parallelism": f"work partition x{world} (one tensor stream per GPU)",
                       "l2": "inputs larger than L2: the lattices (3 directions x 19 planes x 0.94 M pores x "
                             "element, two lattices in the default forms: 431 MB fp32, 216 MB 16-bit) exceed the "
                             "126 MB L2 and stream from HBM every step; a bench step is a whole tensor solve"},
            "glups_fluid": gf, "glups_all_node": ga,
            "steps_per_direction": [r.steps for r in head["runs"]],
            "rel_err_vs_fp64": head["err"], "rel_err_vs_reference": head["err_ref"],
            "mean_velocity": {"superficial_q": qh.tolist(), "pore_mean_q_over_phi": (qh / phi).tolist(),
                              "porosity": phi, "rows": "forcing direction x, y, z; columns q_x, q_y, q_z"},
            "paths": paths,
            "plain_fp32": {"value": kt_p, "unit": "k-tensors/hr", "glups_fluid": gf_p, "glups_all_node": ga_p},
            "speedup_vs_plain_fp32": kt / kt_p,
            "fp64_steps_per_direction": steps64,
            "reference_steps_per_direction": ref["steps"] if ref is not None else None,
            "serving": serving, "large": large, "batch": batch, "plain64": plain64, "perm2d": perm2d,
            "e2e": {"value": kt_e, "unit": "k-tensors/hr", "h2d_bytes_per_step": int(N),
                    "d2h_bytes_per_step": int(3 * 64)},
            # step launches, the deferred reduction, controller and step-base
            # kernels of every 64-launch graph chunk, and the 8 set-up kernels
            # of each solve (mask packing, rank tables, records, 3 lattices)
            "gpu_launches": int(head["launches"] + 3 * (head["launches"] // 64) + 8 * args.steps),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": traffic, "alg_bytes_per_launch": per_launch_alg,
                         "traffic_source": str(TRAFFIC.relative_to(ROOT)) if traffic is not None else None,
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
    """The uneven-size mix: the first `count` structures of the seeded
    256-structure mix (edges from {48,64,96,128,160}; the generator draws
    them in order, so they are the same structures), three directions each,
    solved (a) one structure at a time with plain FP32 per-step launches, (b)
    all resident in one batch (CUDA-graph chunks, per-solve retirement) for
    each batched path.  Reports k-tensors/hour."""
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

    out = {"workload": f"first {args.count} structures of the 256-structure batch mix (edges 48..160, "
                       f"3 directions each)",
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


PLAIN64_ROW = ROOT / "tests" / "golden" / "configs" / "plain64.csv"


def run_plain64_leg(args, device=0):
    """The plain single-solve configuration: the 64^3 sphere packing (r = 6,
    phi 0.60, seed 0), FP64 (the reference's arithmetic), g = 1e-6 (--ff 4),
    lag 1000, eps 1e-6, max 50000 and the reference's other defaults, the
    three forcing directions the reference binary runs.  Device time per
    tensor with CUDA events (autotuned FP64 variant, structure resident), the
    outputs the configuration names (superficial q_x, pore mean q_x / phi,
    k_xx) and every K_ij against the row the reference binary wrote for this
    structure, and the reference binary on all host cores (a bounded
    fixed-step sample scaled by its own step counts)."""
    import torch
    from flow_anizotropy_b200 import _lib
    from flow_anizotropy_b200 import solver as S
    from flow_anizotropy_b200 import structures as st
    import hashlib
    solid = st.plain_64(0)
    ref = reference_row(PLAIN64_ROW)
    if ref is not None and hashlib.sha256(np.ascontiguousarray(solid).tobytes()).hexdigest() != ref["sha256"]:
        ref = None
    F = 2.5e-7 * 4
    forces = [[F, 0, 0], [0, F, 0], [0, 0, F]]
    mu = (1.0 / 3.0) * (1.0 - 0.5)
    phi = float((solid == 0).mean())
    best, _ = S.tune3d(solid, ndir=3, precision="fp64", nsteps=100, device=device)
    p = S.Params3D(precision="fp64", tau=1.0, eps=1e-6, lag=1000, max_steps=50000, variant=best)
    dev = torch.from_numpy(np.ascontiguousarray(solid)).cuda(device)
    ctx = _lib.context(device)
    S.solve3d(dev, forces, p, device=device)
    reps = max(1, args.plain64_reps)
    with EventTimer(torch, ctx.stream) as t:
        for _ in range(reps):
            runs, rc, _ = S.solve3d(dev, forces, p, device=device)
    sec = t.ms / 1e3 / reps
    K = tensor_K(runs, mu, F)
    out = {"workload": "64^3 sphere packing r=6 phi=0.60 seed 0, FP64, 3 directions, g=1e-6, lag 1000, eps 1e-6",
           "kernel_variant": best, "seconds_per_tensor": sec, "k_tensors_per_hr": 3600.0 / sec,
           "steps_per_direction": [r.steps for r in runs], "converged": [r.converged for r in runs],
           "superficial_q_x": float(runs[0].q[0]), "pore_mean_q_x": float(runs[0].q[0] / phi),
           "porosity": phi, "k_xx": float(K[0, 0])}
    if ref is not None:
        cpu = cpu_sample(solid, dict(ff=4.0, tau=1.0), seconds_target=min(args.cpu_seconds, 6.0))
        ent = cpu_baseline_entry(cpu, solid.size, ref["steps"], f"the reference's own run ({ref['path']})")
        out.update({"reference_steps_per_direction": ref["steps"],
                    "steps_equal_reference": [r.steps for r in runs] == ref["steps"],
                    "rel_err_vs_reference": k_errors(K, ref["K"]),
                    "q_rel_err_vs_reference": float(np.abs(np.array([r.q for r in runs]) - ref["q"]).max()
                                                    / np.abs(ref["q"]).max()),
                    "reference_one_core_seconds_recorded": ref["seconds"],
                    "cpu_baseline": ent})
    return out


def run_large_workload(args, device=0):
    """The large configuration: 512^3 Gaussian random field (sigma (3, 3, 9),
    phi = 0.15, largest cluster spanning z), tau = 0.8, three directions
    resident; a fixed number of steps (--large-steps) per storage precision,
    timed with CUDA events with the library's default kernels: fluid GLUPS and the
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
        # the library's default kernels (tuned on the 128^3 workload): timing
        # every variant at this size would cost minutes of the bench
        best = -1
        p = S.Params3D(tau=0.8, eps=0.0, lag=10**9, hold=10**6, min_steps=0, max_steps=args.large_steps,
                       avg_steps=0, precision=prec, criterion="drift", variant=best)
        S.solve3d(dev, forces, S.Params3D(**{**p.__dict__, "max_steps": 20}), device=device)
        with Clocks(device) as clk, EventTimer(torch, ctx.stream) as t:
            runs, _, _ = S.solve3d(dev, forces, p, device=device)
        upd = 3.0 * npore * args.large_steps
        ab = 3.0 * args.large_steps * alg_bytes_per_dir_step(prec, npore, N)
        out["paths"][prec] = {"ms": t.ms, "glups_fluid": upd / (t.ms / 1e3) / 1e9, "kernel_variant": "library default",
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


# ------------------------------------------------------ fixed-step runs ----
STEP_STRUCTURES = {"tensor128": "precision_128", "plain64": "plain_64"}


def run_steps_workload(args, device=0):
    """A fixed number of steps of one precision and kernel variant on a named
    structure, all three forcing directions together (no convergence stop, no
    averaging): the command the kernel profiles in profiles/ capture.  With
    --images N it runs N 256^2 D2Q9 disc packings, both directions, instead."""
    from flow_anizotropy_b200 import solver as S
    from flow_anizotropy_b200 import structures as st
    if args.images > 0:
        imgs = np.stack([st.disc_packing_2d(seed=i, solid_fraction=0.2 + 0.05 * (i % 5)) for i in range(args.images)])
        p2 = S.Params2D(tau=args.tau, lag=args.steps + 1, min_steps=args.steps + 1, max_steps=args.steps, avg_steps=0)
        runs, _ = S.solve2d_many(imgs, [[S.FX_BASE, 0.0], [0.0, S.FX_BASE]], p2, device=device)
        return {"workload": f"D2Q9 {args.images} images x 2 directions, {args.steps} steps",
                "steps": [[r.steps for r in rr] for rr in runs[:2]]}
    solid = getattr(st, STEP_STRUCTURES[args.structure])(0)
    prec = "fp32" if args.precision == "auto" else args.precision
    variant = args.variant
    if variant < 0:
        variant, _ = S.tune3d(solid, ndir=3, precision=prec, nsteps=50, device=device)
    F = 1e-6
    p = S.Params3D(precision=prec, criterion="drift", tau=args.tau, lag=args.lag, max_steps=args.steps,
                   avg_steps=0, hold=10**6, variant=variant)
    runs, _, _ = S.solve3d(solid, [[F, 0, 0], [0, F, 0], [0, 0, F]], p, device=device)
    return {"workload": f"{args.structure} fixed steps", "precision": prec, "variant": variant,
            "steps": [r.steps for r in runs], "q": [list(map(float, r.q)) for r in runs]}


# -------------------------------------------------------- reference arm ----
def run_reference(args, rank, world):
    """The reference CPU solver (oracle/_ref/lbm3d-perm, built from
    LMB3d/lbm3d-perm.cpp with its own flags) on all host cores, one process
    per core as scripts/solve_permeability3d.py runs it.  Each bench step is
    one bounded fixed-step sample of the workload structure (every process
    solves the three directions for a few steps); `steps` and `ms_per_step`
    are those samples as timed.  `value` turns the measured all-node rate into
    converged k-tensors/hour with the step counts the reference itself took
    on this structure (tests/golden/configs/precision128.csv; a full
    converged tensor takes the reference about an hour per core), and says so
    in `extrapolated`."""
    if rank != 0:
        return None
    from flow_anizotropy_b200 import structures as st
    wl = dict(WORKLOAD)
    ref = reference_row()
    if ref is None:
        return {"impl": "reference", "unavailable": f"no reference row at {REF_ROW.relative_to(ROOT)}"}
    solid = st.ellipsoid_packing(wl["n"], wl["semi"], wl["porosity"], wl["seed"])
    N = solid.size
    samples = []
    for i in range(args.warmup + args.steps):
        cpu = cpu_sample(solid, wl, seconds_target=args.cpu_seconds)
        if i >= args.warmup:
            samples.append(cpu)
    lups = statistics.median(c["lups_per_core"] for c in samples)
    cpu = dict(samples[-1], lups_per_core=lups)
    entry = cpu_baseline_entry(cpu, N, ref["steps"], f"the reference's own run ({ref['path']})")
    sample_ms = 1e3 * statistics.mean(c["seconds"] for c in samples)
    return {"metric": METRIC, "value": entry["value"], "unit": "k-tensors/hr", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": sample_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded structure)",
            "config": {"workload": wl["workload"], "seed": wl["seed"], "precision": "fp64",
                       "step": "one fixed-step sample on all host cores (" + cpu["sample"] + ")"},
            "impl": "reference",
            "extrapolated": {"value_from": "median all-node LUPS per core of the timed samples",
                             "formula": entry["formula"], "steps_per_tensor": ref["steps"],
                             "steps_source": entry["steps_source"],
                             "converged_tensor_seconds_per_core": N * float(sum(ref["steps"])) / lups},
            "cpu_baseline": entry,
            "e2e": {"value": entry["value"], "unit": "k-tensors/hr", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="auto", choices=["auto", "fp16", "bf16", "fp32", "fp64", "m32", "md32"])
    ap.add_argument("--serve-seconds", type=float, default=120.0,
                    help="arrival window of the serving leg (0: no serving leg)")
    ap.add_argument("--serve-precision", default="fp16", choices=["fp32", "fp16", "bf16"])
    ap.add_argument("--serve-sustained", type=float, default=0.7,
                    help="serving: second trace at this fraction of the served rate, run to completion (0: none)")
    ap.add_argument("--serve-variant", type=int, default=-1,
                    help="step-kernel variant of the serving batch (-1: library default)")
    ap.add_argument("--serve-pool", type=int, default=40, help="distinct batch-mix structures the requests draw")
    ap.add_argument("--serve-plain-sample", type=int, default=10,
                    help="structures of the plain FP32 one-at-a-time comparison")
    ap.add_argument("--workload", default="tensor128",
                    choices=["tensor128", "batch", "gen3d", "large", "perm2d", "steps"])
    ap.add_argument("--structure", default="tensor128", choices=sorted(STEP_STRUCTURES),
                    help="structure of the steps workload")
    ap.add_argument("--variant", type=int, default=-1, help="steps workload: step-kernel variant (-1: autotune)")
    ap.add_argument("--tau", type=float, default=1.0, help="steps workload: relaxation time")
    ap.add_argument("--lag", type=int, default=10**9,
                    help="steps workload: reduce the flux every LAG steps (1: every step, as in the averaging phase)")
    ap.add_argument("--images", type=int, default=0, help="steps workload: D2Q9 images instead of a 3D structure")
    ap.add_argument("--group2d", type=int, default=16, help="images per launch of the perm2d workload")
    ap.add_argument("--large-n", type=int, default=512, help="cell edge of the large workload")
    ap.add_argument("--large-steps", type=int, default=2000, help="fixed steps of the large leg (0: no large leg)")
    ap.add_argument("--perm2d-images", type=int, default=16,
                    help="D2Q9 leg: seeded 256^2 images solved to convergence, both directions (0: no leg)")
    ap.add_argument("--plain64-reps", type=int, default=3,
                    help="timed 64^3 FP64 single-solve tensors (the plain configuration; 0: no leg)")
    ap.add_argument("--gen-size", type=int, default=80, help="cell edge of the gen3d workload")
    ap.add_argument("--count", type=int, default=48,
                    help="structures of the batch leg / workload (0: no batch leg)")
    ap.add_argument("--batch-paths", default="fp16")
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
    elif args.workload == "steps":
        out = run_steps_workload(args, local_rank) if rank == 0 else None
    else:
        out = run_ours(args, rank, world, local_rank)
    if out is not None and rank == 0:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
