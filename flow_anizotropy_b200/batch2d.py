"""Solve a generated 2D structure set on one GPU, many images per launch.

Driver-side batching for ``scripts/solve_permeability.py`` datasets: instead
of one ``lbm2d-perm`` process per image (``ProcessPoolExecutor`` over
subprocesses, scripts/solve_permeability.py:29-46, 78-95), the images of
``<dataset>/structures.csv`` are read in one process and solved ``--group``
at a time by ``lbm_solve2d_many``: every (image, direction) solve of a group
advances in the same launch per step, each with its own mask and controller,
so each result equals the drop-in solving that image alone.

Each image's row (the drop-in's header, columns and number format, with the
image path as ``filename``) goes to ``<dataset>/perm/<sample_id:06d>.csv``,
written to a temporary name and renamed when complete; images whose CSV
already holds a row are skipped, so a rerun resumes.  ``--extra`` takes the
flags the driver would pass to the solver (``--eps``, ``--size`` ...); the
reference driver's ``--merge-only`` then joins the rows onto structures.csv
unchanged:

    python -m flow_anizotropy_b200.batch2d --dataset DATA/aniso --ff 1
    python scripts/solve_permeability.py --dataset DATA/aniso --merge-only
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

from . import cli2d
from . import solver as S
from . import tensor as T
from .batch3d import Task, plan
from .structure_io import load_structure2d


def solver_config(extra: str):
    """cli2d's option set from the driver's --extra string."""
    parsed = cli2d.parse(["structure", "out.csv"] + extra.split())
    if parsed is None:
        raise SystemExit("--help in --extra")
    cfg = parsed[2]
    if cfg["velocity"]:
        raise SystemExit("--velocity is not supported in batch mode (use the lbm2d-perm drop-in)")
    return cfg


def done(task: Task) -> bool:
    """The reference driver's cache rule: the CSV exists and is not empty
    (scripts/solve_permeability.py:30-31)."""
    return os.path.exists(task.out_csv) and os.path.getsize(task.out_csv) > 0


def write_row(task: Task, cfg, solid, rx, ry) -> int:
    """The drop-in's row for one image, moved into place atomically; returns
    the drop-in's exit code (0 converged, 3 kept but flagged)."""
    ny, nx = solid.shape
    F = S.FX_BASE * cfg["ff"]
    mu = cli2d.mu_2d(cfg["tau"])
    nfluid = int((solid == 0).sum())
    porosity = float(np.float32(nfluid) / np.float32(nx * ny))
    Tn = T.assemble2(rx, ry, mu, F)
    row = T.row2(task.structure, cfg["ff"], F, mu, porosity, rx, ry, Tn)
    tmp = f"{task.out_csv}.tmp.{os.getpid()}"
    try:
        if os.path.exists(tmp):
            os.remove(tmp)
        T.append_csv(tmp, T.header2(), row)
        os.replace(tmp, task.out_csv)
    finally:
        if os.path.exists(tmp):
            os.remove(tmp)
    return 0 if (rx.converged and ry.converged) else 3


def run(dataset, ff=1.0, limit=0, extra="", group=16, device=0, log=print):
    """Solve every missing image; returns dict(solved, cached, unconverged, failed=[(id, msg)])."""
    cfg = solver_config(extra)
    cfg["ff"] = ff
    tasks = plan(dataset, limit)
    os.makedirs(os.path.join(dataset, "perm"), exist_ok=True)
    work = [t for t in tasks if not done(t)]
    out = {"solved": 0, "cached": len(tasks) - len(work), "unconverged": 0, "failed": []}
    log(f"{len(tasks)} structures: {out['cached']} already solved, {len(work)} to do")
    F = S.FX_BASE * ff
    forces = [[F, 0.0], [0.0, F]]
    params = S.Params2D(tau=cfg["tau"], eps=cfg["eps"], lag=cfg["lag"], hold=cfg["hold"],
                        min_steps=cfg["min_steps"], max_steps=cfg["max_steps"], avg_steps=cfg["avg_steps"],
                        avg_sample=cfg["avg_sample"], qfloor=cfg["qfloor"], ksigma=cfg["ksigma"])
    nx, ny = cfg["size"]
    batch: list[tuple[Task, np.ndarray]] = []

    def flush():
        if not batch:
            return
        solids = np.stack([s for _, s in batch])
        try:
            runs, _ = S.solve2d_many(solids, forces, params, device=device)
        except S.LBMError as e:
            for t, _ in batch:
                out["failed"].append((t.sample_id, str(e)))
            batch.clear()
            return
        for (t, solid), (rx, ry) in zip(batch, runs):
            if rx.status or ry.status:
                out["failed"].append((t.sample_id, "non-finite flux"))
                continue
            try:
                rc = write_row(t, cfg, solid, rx, ry)
            except OSError as e:
                out["failed"].append((t.sample_id, f"cannot write {t.out_csv}: {e}"))
                continue
            out["solved"] += 1
            out["unconverged"] += rc == 3
        batch.clear()

    for t in work:
        try:
            solid = np.ascontiguousarray(load_structure2d(t.structure, nx, ny), dtype=np.uint8)
        except Exception as e:                 # noqa: BLE001 - reported per image
            out["failed"].append((t.sample_id, f"cannot read {t.structure}: {e}"))
            continue
        if solid.max(initial=0) > 1 or not (solid == 0).any():
            out["failed"].append((t.sample_id, "structure has no pore space or non-binary values"))
            continue
        if batch and solid.shape != batch[0][1].shape:
            flush()
        batch.append((t, solid))
        if len(batch) >= group:
            flush()
    flush()
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--dataset", required=True, help="directory with structures.csv and structures/")
    ap.add_argument("--ff", type=float, default=1.0)
    ap.add_argument("--limit", type=int, default=0, help="solve only the first N")
    ap.add_argument("--extra", default="", help='solver flags, e.g. "--eps 5e-4 --size 128x128"')
    ap.add_argument("--group", type=int, default=16, help="images per launch")
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    if not os.path.exists(os.path.join(a.dataset, "structures.csv")):
        sys.exit(f"no structures.csv in {a.dataset}")
    res = run(a.dataset, ff=a.ff, limit=a.limit, extra=a.extra, group=a.group, device=a.device)
    print(f"solved {res['solved']}   cached {res['cached']}   non-converged (kept, flagged) "
          f"{res['unconverged']}   failed {len(res['failed'])}")
    for sid, msg in res["failed"][:10]:
        print(f"  {sid:06d}: {msg}")
    return 1 if res["failed"] else 0


if __name__ == "__main__":
    sys.exit(main())
