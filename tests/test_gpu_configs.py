"""GPU solves of the benchmark configurations against rows the REFERENCE wrote.

tests/golden/configs/<name>.csv is the row the reference binary (built from
LMB3d/lbm3d-perm.cpp with its own flags) appended for the seeded structure
named in <name>.json, with that file's argv (tests/golden/make_golden_configs.py
wrote both).  The structure is rebuilt here from its generator and seed and
must hash to the recorded SHA-256, so the GPU solves exactly the bytes the
reference solved.

  plain64       64^3 sphere packing, phi 0.60 (the single-solve configuration)
  precision128  128^3 prolate-ellipsoid packing, phi 0.45 (the precision study
                the benchmark times)

Tolerances, per tensor entry K_ij = mu q_i^(j) / F
(LMB3d/lbm3d-perm.cpp:522-529) and per mean-velocity component:
  FP64 1e-8, FP32 1e-4, FP16 / BF16 shifted storage 1e-3,
relative to the entry for the diagonal and the flux along the force, and to
the largest diagonal entry (largest flux component) for the off-diagonal ones,
which are differences of nearly cancelling sums and ~1e-3 of the diagonal
here.  FP64 also keeps the reference's step counts and convergence flags
exactly (same stopping rule, same arithmetic up to the reference's
-ffast-math roundoff).  The reduced-precision paths stop by their own
criterion (batch-means block test for FP16 / BF16), so their step counts are
not compared.
"""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

from flow_anizotropy_b200 import solver as S
from flow_anizotropy_b200 import structures as st
from flow_anizotropy_b200 import tensor as T

C = Path(__file__).resolve().parent / "golden" / "configs"
NAMES = sorted(p.stem for p in C.glob("*.json")) if C.exists() else []
TOL = {"fp64": 1e-8, "fp32": 1e-4, "fp16": 1e-3, "bf16": 1e-3}
TAGS = ("fx", "fy", "fz")


def load(name):
    meta = json.loads((C / f"{name}.json").read_text())
    lines = (C / f"{name}.csv").read_text().splitlines()
    assert lines[0] == T.header3()
    row = dict(zip(lines[0].split(","), lines[1].split(",")))
    return meta, row


def knobs(argv):
    p = dict(ff=1.0, eps=1e-5, lag=2000, hold=2, min_steps=4000, max_steps=200000, avg_steps=2000)
    key = {"--ff": "ff", "--eps": "eps", "--lag": "lag", "--hold": "hold", "--min-steps": "min_steps",
           "--max-steps": "max_steps", "--avg-steps": "avg_steps"}
    for a, v in zip(argv[::2], argv[1::2]):
        p[key[a]] = float(v) if a in ("--ff", "--eps") else int(v)
    return p


def structure(meta):
    s = getattr(st, meta["generator"])(meta["seed"])
    assert hashlib.sha256(s.tobytes()).hexdigest() == meta["sha256"], "generator no longer reproduces the structure"
    return s


def k_matrix_errors(K, Kref):
    """|K_ij - Kref_ij| relative to |Kref_ij| on the diagonal and to max|Kref_ii| off it."""
    scale = np.abs(np.diag(Kref)).max()
    err = np.abs(K - Kref)
    den = np.where(np.eye(3, dtype=bool), np.abs(Kref), scale)
    return err / den


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64", "fp32", "fp16", "bf16"])
@pytest.mark.parametrize("name", NAMES)
def test_config_tensor_matches_reference(gpu, name, prec):
    meta, row = load(name)
    solid = structure(meta)
    kn = knobs(meta["argv"])
    F = S.FX_BASE * kn["ff"]
    mu = S.nu_of_tau(1.0)
    p = S.Params3D(eps=kn["eps"], lag=kn["lag"], hold=kn["hold"], min_steps=kn["min_steps"],
                   max_steps=kn["max_steps"], avg_steps=kn["avg_steps"], precision=prec)
    runs, rc, _ = S.solve3d(solid, [[F, 0, 0], [0, F, 0], [0, 0, F]], p)
    qref = np.array([[float(row[f"q{c}_{t}"]) for c in "xyz"] for t in TAGS])     # [direction][component]
    q = np.array([r.q for r in runs])
    if prec == "fp64":
        assert [r.steps for r in runs] == [int(row[f"steps_{t}"]) for t in TAGS]
        assert [r.converged for r in runs] == [int(row[f"conv_{t}"]) for t in TAGS]
        assert rc == (0 if all(int(row[f"conv_{t}"]) for t in TAGS) else 3)
    tol = TOL[prec]
    # mean velocity: superficial q (the reference's output) and the pore mean
    # q / phi, per component, against the flux along the force
    phi = float((solid == 0).mean())
    assert abs(phi - float(row["porosity"])) < 1e-9
    for j in range(3):
        scale = np.abs(qref[j]).max()
        assert np.all(np.abs(q[j] - qref[j]) <= tol * scale), (TAGS[j], q[j], qref[j])
        assert np.all(np.abs(q[j] / phi - qref[j] / phi) <= tol * scale / phi)
    K = np.array([[mu * q[j][c] / F for j in range(3)] for c in range(3)])
    Kref = np.array([[float(row[f"K_{a}{b}"]) for b in "xyz"] for a in "xyz"])
    e = k_matrix_errors(K, Kref)
    assert e.max() <= tol, (prec, e)
