"""Solve a generated 3D structure set on one GPU through the resident batch.

Driver-side batching for ``scripts/solve_permeability3d.py`` datasets: instead
of one solver process per structure (``--solver`` + ``ProcessPoolExecutor``,
scripts/solve_permeability3d.py:250-259), every structure of
``<dataset>/structures.csv`` is submitted to one continuous-batching server
(``flow_anizotropy_b200.serve.Server``), which keeps many solves resident on
the device and admits the next structure as soon as one retires.

The outputs are exactly the per-sample files the reference driver produces
and merges: ``<dataset>/perm/<sample_id:06d>.csv`` holding the CSV header and
one row of the ``lbm3d-perm`` drop-in (same columns, same number format, the
structure path as ``filename``), each written to ``<out>.tmp.<pid>`` and
renamed into place only when complete (scripts/solve_permeability3d.py:120-144).
A sample whose CSV is already complete is skipped and an incomplete one is
redone (the driver's ``valid_result`` rule, :88-106), so a killed run resumes
where it stopped.  ``--shard I/N``, ``--interleave COL``, ``--limit`` and
``--ff`` mean what they mean for the driver; ``--extra`` takes the solver
flags the driver would pass (``--eps``, ``--lag``, ``--validate``, ...).
Afterwards the reference driver builds permeability.csv unchanged:

    python -m flow_anizotropy_b200.batch3d --dataset DATA/aniso3d --extra "--precision fp32"
    python scripts/solve_permeability3d.py --dataset DATA/aniso3d --merge-only

Results are those of the drop-in solving each structure alone (a batched
solve is bit-identical to the same solve alone).
"""
from __future__ import annotations

import argparse
import math
import os
import queue
import sys
import threading
from dataclasses import dataclass

import numpy as np

from . import cli3d
from . import solver as S
from . import tensor as T
from .structure_io3d import read_raw_checked

# Columns a finished per-sample CSV must carry (scripts/solve_permeability3d.py:82-83).
REQUIRED_COLS = ("K_xx", "K_yy", "K_zz", "k_xy", "k_xz", "k_yz", "conv_fx", "conv_fy", "conv_fz")


def valid_result(path) -> bool:
    """A complete solve: one data row with finite tensor columns and the three
    convergence flags (the driver's cache test, scripts/solve_permeability3d.py:88-106)."""
    import pandas as pd
    try:
        if os.path.getsize(path) <= 0:
            return False
        one = pd.read_csv(path)
    except Exception:
        return False
    if len(one) < 1 or not set(REQUIRED_COLS) <= set(one.columns):
        return False
    return bool(np.isfinite(one[list(REQUIRED_COLS)].to_numpy(float)).all())


@dataclass
class Task:
    sample_id: int
    structure: str       # path as the driver passes it to the solver (the CSV's filename)
    out_csv: str


def plan(dataset, limit=0, shard="", interleave=""):
    """The driver's task list: structures.csv rows (first `limit`), the shard
    I/N subset (sample_id % N == I), in round-robin order over `interleave`."""
    import pandas as pd
    df = pd.read_csv(os.path.join(dataset, "structures.csv"))
    if limit:
        df = df.head(limit)
    if shard:
        si, sn = (int(v) for v in shard.split("/"))
        if not 0 <= si < sn:
            raise SystemExit(f"bad --shard {shard}")
        df = df[df.sample_id % sn == si].reset_index(drop=True)
    order = df
    if interleave:
        rank = df.groupby(interleave, sort=False).cumcount()
        order = df.assign(_r=rank).sort_values(["_r", interleave], kind="stable")
    perm_dir = os.path.join(dataset, "perm")
    structures_dir = os.path.join(dataset, "structures")
    return [Task(int(r.sample_id), os.path.join(structures_dir, r.filename),
                 os.path.join(perm_dir, f"{int(r.sample_id):06d}.csv")) for r in order.itertuples()]


def todo(tasks):
    """Split tasks into (to solve, cached); incomplete CSVs are removed."""
    work, cached = [], []
    for t in tasks:
        if os.path.exists(t.out_csv):
            if valid_result(t.out_csv):
                cached.append(t)
                continue
            os.remove(t.out_csv)          # a killed run: redo it rather than inherit it
        work.append(t)
    return work, cached


def solver_config(extra: str, precision: str | None):
    """cli3d's option set from the driver's --extra string."""
    argv = ["structure", "out.csv"] + extra.split()
    if precision and "--precision" not in argv:
        argv += ["--precision", precision]
    _, _, cfg = cli3d.parse(argv)
    if cfg["velocity"]:
        raise SystemExit("--velocity is not supported in batch mode (use the lbm3d-perm drop-in)")
    return cfg


def write_row(task: Task, cfg, solid, runs) -> int:
    """Assemble the drop-in's CSV row and move it into place atomically;
    returns the drop-in's exit code (0 converged, 3 kept but flagged)."""
    nz, ny, nx = solid.shape
    porosity = int((solid == 0).sum()) / float(solid.size)
    F = S.FX_BASE * cfg["ff"]
    mu = (1.0 / 3.0) * (cfg["tau"] - 0.5)
    rx, ry, rz = runs[:3]
    Tn = T.assemble3([rx.q, ry.q, rz.q], mu, F)
    row = T.row3(task.structure, cfg["ff"], F, mu, (nx, ny, nz), porosity, [rx, ry, rz], Tn)
    tmp = f"{task.out_csv}.tmp.{os.getpid()}"
    try:
        if os.path.exists(tmp):
            os.remove(tmp)
        T.append_csv(tmp, T.header3(), row)
        if not valid_result(tmp):
            raise OSError("incomplete row")
        os.replace(tmp, task.out_csv)
    finally:
        if os.path.exists(tmp):
            os.remove(tmp)
    return 0 if (rx.converged and ry.converged and rz.converged) else 3


def run(dataset, ff=1.0, limit=0, shard="", interleave="", extra="", precision=None,
        hbm_budget=150 * 2**30, max_work=None, chunk=256, device=0, prefetch=8, log=print):
    """Solve every missing sample; returns dict(solved, cached, unconverged, failed=[(id, msg)])."""
    from .serve import Server
    cfg = solver_config(extra, precision)
    cfg["ff"] = ff
    tasks = plan(dataset, limit, shard, interleave)
    os.makedirs(os.path.join(dataset, "perm"), exist_ok=True)
    work, cached = todo(tasks)
    log(f"{len(tasks)} structures: {len(cached)} already solved, {len(work)} to do")
    F = S.FX_BASE * ff
    forces = [[F, 0, 0], [0, F, 0], [0, 0, F]]
    if cfg["validate"]:
        c = 1.0 / math.sqrt(3.0)
        forces.append([F * c, F * c, F * c])
    params = S.Params3D(tau=cfg["tau"], eps=cfg["eps"], lag=cfg["lag"], hold=cfg["hold"],
                        min_steps=cfg["min_steps"], max_steps=cfg["max_steps"],
                        avg_steps=cfg["avg_steps"], precision=cfg["precision"],
                        criterion=cfg["criterion"])
    out = {"solved": 0, "cached": len(cached), "unconverged": 0, "failed": []}
    if not work:
        return out

    # structures are read ahead on a host thread while the device solves
    loaded: queue.Queue = queue.Queue(maxsize=max(1, prefetch))

    def reader():
        for t in work:
            try:
                loaded.put((t, read_raw_checked(t.structure), None))
            except BaseException as e:          # noqa: BLE001 - reported per sample
                loaded.put((t, None, str(e)))
        loaded.put(None)

    th = threading.Thread(target=reader, daemon=True)
    th.start()
    kw = {} if max_work is None else {"max_work": max_work}
    srv = Server(precision=cfg["precision"], hbm_budget=hbm_budget, chunk=chunk, device=device, **kw)
    pending: dict[int, tuple[Task, np.ndarray]] = {}
    reading = True
    try:
        while reading or not srv.idle():
            # keep a few structures queued in the server beyond what is resident
            while reading and len(srv.queue) < 2:
                item = loaded.get()
                if item is None:
                    reading = False
                    break
                t, solid, err = item
                if err is not None:
                    out["failed"].append((t.sample_id, err))
                    continue
                rid = srv.submit(solid, forces, params)
                pending[rid] = (t, solid)
            if srv.idle():
                continue
            srv.pump()
            for rid in [r for r in srv.finished if r in pending]:
                t, solid = pending.pop(rid)
                req = srv.finished.pop(rid)
                if req.error is not None:
                    out["failed"].append((t.sample_id, req.error))
                    continue
                runs = req.results
                bad = [r for r in runs if r.status]
                if bad:
                    out["failed"].append((t.sample_id, f"non-finite flux at step {bad[0].steps}"))
                    continue
                try:
                    rc = write_row(t, cfg, solid, runs)
                except OSError as e:
                    out["failed"].append((t.sample_id, f"cannot write {t.out_csv}: {e}"))
                    continue
                out["solved"] += 1
                out["unconverged"] += rc == 3
    finally:
        srv.close()
    th.join(timeout=5)
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--dataset", required=True, help="directory with structures.csv and structures/")
    ap.add_argument("--ff", type=float, default=1.0)
    ap.add_argument("--limit", type=int, default=0, help="solve only the first N")
    ap.add_argument("--shard", default="", help="I/N: only samples with sample_id %% N == I")
    ap.add_argument("--interleave", default="", help="solve order round-robin over this column")
    ap.add_argument("--extra", default="", help='solver flags, e.g. "--eps 1e-6 --lag 1000 --validate"')
    ap.add_argument("--precision", default=None,
                    help="storage precision unless --extra names one (default: the drop-in's fp64)")
    ap.add_argument("--hbm-budget-gb", type=float, default=150.0)
    ap.add_argument("--chunk", type=int, default=256, help="steps per CUDA-graph launch")
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    if not os.path.exists(os.path.join(a.dataset, "structures.csv")):
        sys.exit(f"no structures.csv in {a.dataset}")
    res = run(a.dataset, ff=a.ff, limit=a.limit, shard=a.shard, interleave=a.interleave, extra=a.extra,
              precision=a.precision, hbm_budget=int(a.hbm_budget_gb * 2**30), chunk=a.chunk, device=a.device)
    print(f"solved {res['solved']}   cached {res['cached']}   non-converged (kept, flagged) "
          f"{res['unconverged']}   failed {len(res['failed'])}")
    for sid, msg in res["failed"][:10]:
        print(f"  {sid:06d}: {msg}")
    return 1 if res["failed"] else 0


if __name__ == "__main__":
    sys.exit(main())
