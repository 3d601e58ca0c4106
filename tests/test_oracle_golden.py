"""Pin the CPU oracle to the reference: the golden fixtures in tests/golden/
are CSV rows written by the reference binaries (built from the reference
sources by oracle/build_ref.sh, generated by tests/golden/make_golden.py).
The oracle must reproduce step counts and convergence flags exactly and every
number to the 10 printed digits; the host tensor assembly (tensor.row3/row2)
fed with the oracle's fluxes must reproduce the whole row."""
import json
import math
from pathlib import Path

import numpy as np
import pandas as pd
import pytest

from flow_anizotropy_b200 import tensor as T
from flow_anizotropy_b200.cli2d import mu_2d
from flow_anizotropy_b200.structure_io import load_dat
from flow_anizotropy_b200.structure_io3d import load_structure
from oracle import oracle as O
from rowcheck import argv_params, close_row  # noqa: F401

G = Path(__file__).resolve().parent / "golden"
META = json.loads((G / "golden.json").read_text())


@pytest.mark.parametrize("name", [n for n in META if n.startswith("case3d")])
def test_oracle3d_reproduces_reference(name):
    m = META[name]
    tau = 0.8 if m["binary"].endswith("tau0.8") else 1.0
    p, flags = argv_params(m["argv"], dict(O.DEF3D, ff=1.0))
    ff = p.pop("ff")
    p["tau"] = tau
    solid = load_structure(G / f"{name}.raw")
    ref = pd.read_csv(G / f"{name}.csv", dtype=str)
    row_ref = (G / f"{name}.csv").read_text().splitlines()[1]
    F = 2.5e-7 * ff
    runs = []
    qref = np.array([[float(ref[f"q{c}_{t}"][0]) for c in "xyz"] for t in ("fx", "fy", "fz")])
    qscale = np.abs(qref).max()
    blocked = []
    for j, tag in enumerate(("fx", "fy", "fz")):
        force = [0.0, 0.0, 0.0]
        force[j] = F
        r = O.solve3d(solid, force, **p)
        if np.abs(qref[j]).max() < 1e-10 * qscale:
            # a blocked direction: its flux is roundoff, and so is the step at
            # which the drift test passes; check the flux is zero instead
            assert np.abs(r["q"]).max() < 1e-10 * qscale
            blocked.append(j)
            r = dict(r, steps=int(ref[f"steps_{tag}"][0]), converged=int(ref[f"conv_{tag}"][0]), q=qref[j],
                     se=np.array([float(ref[f"se_q{c}_{tag}"][0]) for c in "xyz"]))
        assert r["steps"] == int(ref[f"steps_{tag}"][0]) and r["converged"] == int(ref[f"conv_{tag}"][0])
        runs.append(type("R", (), dict(q=r["q"], se=r["se"], steps=r["steps"], converged=r["converged"])))
    mu = (1.0 / 3.0) * (tau - 0.5)
    Tn = T.assemble3([r.q for r in runs], mu, F)
    nz, ny, nx = solid.shape
    por = float((solid == 0).sum()) / solid.size
    row = T.row3(f"{name}.raw", ff, F, mu, (nx, ny, nz), por, runs, Tn)
    close_row(row, row_ref, T.header3(), rtol=5e-9)
    assert (G / f"{name}.csv").read_text().splitlines()[0] == T.header3()
    if "validate" in flags:
        c = 1.0 / math.sqrt(3.0)
        rv = O.solve3d(solid, [F * c] * 3, **p)
        pred = [(Tn.Ks[r][0] + Tn.Ks[r][1] + Tn.Ks[r][2]) * F * c / mu for r in range(3)]
        line = [s for s in m["stdout"] if "measured" in s][0]
        meas = [float(v) for v in line.split("(")[1].rstrip(")").split(",")]
        np.testing.assert_allclose(rv["q"], meas, rtol=1e-5)
        np.testing.assert_allclose(pred, rv["q"], rtol=1e-6)


def test_oracle2d_reproduces_reference():
    name = "case2d_a"
    m = META[name]
    p, flags = argv_params(m["argv"], dict(O.DEF2D, ff=1.0))
    ff = p.pop("ff")
    val = p.pop("validate", None)
    solid = load_dat(G / f"{name}.dat")
    ref = pd.read_csv(G / f"{name}.csv", dtype=str)
    row_ref = (G / f"{name}.csv").read_text().splitlines()[1]
    F = 2.5e-7 * ff
    rx = O.solve2d(solid, [F, 0.0], **p)
    ry = O.solve2d(solid, [0.0, F], **p)
    for r, tag in ((rx, "fx"), (ry, "fy")):
        assert r["steps"] == int(ref[f"steps_{tag}"][0]) and r["converged"] == int(ref[f"conv_{tag}"][0])
    mu = mu_2d(1.0)
    wrap = lambda r: type("R", (), dict(q=r["q"], se=r["se"], steps=r["steps"], converged=r["converged"],
                                        fieldres=r["fieldres"]))
    Tn = T.assemble2(wrap(rx), wrap(ry), mu, F)
    por = float(np.float32((solid == 0).sum()) / np.float32(solid.size))
    row = T.row2(f"{name}.dat", ff, F, mu, por, wrap(rx), wrap(ry), Tn)
    # the 2D reference is strict IEEE float: only the FP64 flux sums can differ
    close_row(row, row_ref, T.header2(), rtol=1e-9)
    assert (G / f"{name}.csv").read_text().splitlines()[0] == T.header2()
