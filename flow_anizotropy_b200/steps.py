"""Run a fixed number of solver steps on a named workload (for profiling).

    python -m flow_anizotropy_b200.steps --workload tensor128 --precision fp16 --steps 24
    python -m flow_anizotropy_b200.steps --images 16 --steps 24        # D2Q9, 16 images

Builds the seeded structure, solves the three forcing directions together for
exactly --steps steps (no convergence stop, no averaging) and prints the
fluxes.  `ncu -k regex:step3d -s S -c C` on this command captures step
launches of the same kernels the benchmark runs.
"""
from __future__ import annotations

import argparse

import numpy as np

from . import solver as S
from . import structures as st

WORKLOADS = {
    "tensor128": lambda: st.precision_128(0),
    "plain64": lambda: st.plain_64(0),
}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--workload", default="tensor128", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", default="fp32", choices=["fp64", "fp32", "fp16", "bf16", "m32", "md32"])
    ap.add_argument("--variant", type=int, default=-1, help="step-kernel variant (-1: autotune)")
    ap.add_argument("--steps", type=int, default=24)
    ap.add_argument("--tau", type=float, default=1.0)
    ap.add_argument("--lag", type=int, default=10**9,
                    help="reduce the flux every LAG steps (1: every step, as in the averaging phase)")
    ap.add_argument("--images", type=int, default=0,
                    help="D2Q9 instead: this many 256^2 disc packings, both directions, one launch per step")
    a = ap.parse_args(argv)
    if a.images > 0:
        imgs = np.stack([st.disc_packing_2d(seed=i, solid_fraction=0.2 + 0.05 * (i % 5)) for i in range(a.images)])
        p2 = S.Params2D(tau=a.tau, lag=a.steps + 1, min_steps=a.steps + 1, max_steps=a.steps, avg_steps=0)
        runs, _ = S.solve2d_many(imgs, [[S.FX_BASE, 0.0], [0.0, S.FX_BASE]], p2)
        for rr in runs[:2]:
            print([r.steps for r in rr], [r.q for r in rr])
        return
    solid = WORKLOADS[a.workload]()
    variant = a.variant
    if variant < 0:
        variant, _ = S.tune3d(solid, ndir=3, precision=a.precision, nsteps=50)
    F = 1e-6
    p = S.Params3D(precision=a.precision, criterion="drift", tau=a.tau, lag=a.lag, max_steps=a.steps,
                   avg_steps=0, hold=10**6, variant=variant)
    runs, rc, _ = S.solve3d(solid, [[F, 0, 0], [0, F, 0], [0, 0, F]], p)
    for r in runs:
        print(r.steps, r.q)


if __name__ == "__main__":
    main()
