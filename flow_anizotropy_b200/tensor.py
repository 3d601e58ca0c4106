"""Permeability tensor assembly and the solvers' CSV rows.

3D: LMB3d/lbm3d-perm.cpp:522-553 (K from three solves, symmetrised
off-diagonals, reciprocity residuals, cyclic-Jacobi principal values and
axes, fractional anisotropy) and the CSV of :574-615.
2D: LMB2d/main.cpp:326-353 and the CSV of :383-411.

CSV numbers are printed like a C++ stream with ``setprecision(10)``, i.e.
``%.10g``, so the rows are byte-compatible with the reference binaries'.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass

import numpy as np

AXES = "xyz"
TAGS3 = ("fx", "fy", "fz")


def fmt(v) -> str:
    """A value as ``ostream << setprecision(10)`` prints it."""
    if isinstance(v, (int, np.integer)):
        return str(int(v))
    v = float(v)
    if math.isnan(v):
        return "-nan" if math.copysign(1.0, v) < 0 else "nan"
    if math.isinf(v):
        return "inf" if v > 0 else "-inf"
    return "%.10g" % v


def jacobi3(A):
    """Cyclic Jacobi eigen-decomposition of a symmetric 3x3, as LMB3d/lbm3d-perm.cpp:401-443.

    Returns (val[3] sorted descending, vec[3][3] with eigenvectors in columns).
    """
    a = [[float(A[i][j]) for j in range(3)] for i in range(3)]
    vec = [[1.0 if i == j else 0.0 for j in range(3)] for i in range(3)]
    for _ in range(50):
        off = abs(a[0][1]) + abs(a[0][2]) + abs(a[1][2])
        if off < 1e-18:
            break
        for p in range(2):
            for q in range(p + 1, 3):
                if abs(a[p][q]) < 1e-300:
                    continue
                theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q])
                t = (1.0 if theta >= 0 else -1.0) / (abs(theta) + math.sqrt(theta * theta + 1.0))
                c = 1.0 / math.sqrt(t * t + 1.0)
                s = t * c
                for k in range(3):
                    akp, akq = a[k][p], a[k][q]
                    a[k][p] = c * akp - s * akq
                    a[k][q] = s * akp + c * akq
                for k in range(3):
                    apk, aqk = a[p][k], a[q][k]
                    a[p][k] = c * apk - s * aqk
                    a[q][k] = s * apk + c * aqk
                    vkp, vkq = vec[k][p], vec[k][q]
                    vec[k][p] = c * vkp - s * vkq
                    vec[k][q] = s * vkp + c * vkq
    val = [a[i][i] for i in range(3)]
    for i in range(2):
        for j in range(i + 1, 3):
            if val[j] > val[i]:
                val[i], val[j] = val[j], val[i]
                for k in range(3):
                    vec[k][i], vec[k][j] = vec[k][j], vec[k][i]
    return val, vec


@dataclass
class Tensor3:
    K: list            # K[c][j]: flux component c under force along j
    k_xy: float
    k_xz: float
    k_yz: float
    rec_xy: float
    rec_xz: float
    rec_yz: float
    recip: float
    Ks: list
    val: list
    vec: list
    kmean: float
    fa: float


def assemble3(q_runs, mu, F) -> Tensor3:
    """LMB3d/lbm3d-perm.cpp:522-553.  q_runs[j] is the flux of the solve forced along j."""
    with np.errstate(divide="ignore", invalid="ignore"):
        K = [[float(np.float64(mu) * q_runs[j][c] / np.float64(F)) for j in range(3)]
             for c in range(3)]
    trace = K[0][0] + K[1][1] + K[2][2]
    k_xy = 0.5 * (K[0][1] + K[1][0])
    k_xz = 0.5 * (K[0][2] + K[2][0])
    k_yz = 0.5 * (K[1][2] + K[2][1])

    def rdiv(a, b):
        try:
            return a / b
        except ZeroDivisionError:
            return math.nan if a == 0 else math.copysign(math.inf, a)

    rec_xy = rdiv(abs(K[0][1] - K[1][0]), abs(trace))
    rec_xz = rdiv(abs(K[0][2] - K[2][0]), abs(trace))
    rec_yz = rdiv(abs(K[1][2] - K[2][1]), abs(trace))
    recip = _cmax(rec_xy, _cmax(rec_xz, rec_yz))
    Ks = [[K[0][0], k_xy, k_xz], [k_xy, K[1][1], k_yz], [k_xz, k_yz, K[2][2]]]
    val, vec = jacobi3(Ks)
    kmean = trace / 3.0
    dv = ((val[0] - val[1]) ** 2 + (val[1] - val[2]) ** 2 + (val[2] - val[0]) ** 2)
    nrm = val[0] ** 2 + val[1] ** 2 + val[2] ** 2
    fa = math.sqrt(0.5 * dv / nrm) if nrm > 0 else math.nan
    return Tensor3(K, k_xy, k_xz, k_yz, rec_xy, rec_xz, rec_yz, recip, Ks, val, vec, kmean, fa)


def _cmax(a, b):
    """std::max(a, b): returns a unless a < b (so NaN in a propagates, NaN in b does not)."""
    return b if a < b else a


def header3() -> str:
    cols = ["filename", "ff", "force", "mu", "nx", "ny", "nz", "porosity",
            "steps_fx", "conv_fx", "steps_fy", "conv_fy", "steps_fz", "conv_fz"]
    cols += [f"q{c}_{t}" for t in TAGS3 for c in AXES]
    cols += [f"se_q{c}_{t}" for t in TAGS3 for c in AXES]
    cols += [f"K_{r}{c}" for r in AXES for c in AXES]
    cols += ["k_xy", "k_xz", "k_yz", "recip_xy", "recip_xz", "recip_yz", "recip_resid",
             "k1", "k2", "k3", "k_mean", "fa",
             "v1_x", "v1_y", "v1_z", "v2_x", "v2_y", "v2_z", "v3_x", "v3_y", "v3_z"]
    return ",".join(cols)


def row3(filename, ff, F, mu, shape_xyz, porosity, runs, T: Tensor3) -> str:
    """One CSV row in the column order of LMB3d/lbm3d-perm.cpp:600-614."""
    nx, ny, nz = shape_xyz
    vals = [filename, fmt(ff), fmt(F), fmt(mu), fmt(nx), fmt(ny), fmt(nz), fmt(porosity)]
    for r in runs:
        vals += [fmt(int(r.steps)), fmt(int(r.converged))]
    vals += [fmt(runs[j].q[c]) for j in range(3) for c in range(3)]
    vals += [fmt(runs[j].se[c]) for j in range(3) for c in range(3)]
    vals += [fmt(T.K[r][c]) for r in range(3) for c in range(3)]
    vals += [fmt(v) for v in (T.k_xy, T.k_xz, T.k_yz, T.rec_xy, T.rec_xz, T.rec_yz, T.recip,
                              T.val[0], T.val[1], T.val[2], T.kmean, T.fa)]
    vals += [fmt(T.vec[i][j]) for j in range(3) for i in range(3)]
    return ",".join(str(v) for v in vals)


def append_csv(path, header: str, row: str) -> None:
    """Append a row, writing the header first if the file is empty or absent
    (LMB3d/lbm3d-perm.cpp:575-598)."""
    need_header = not (os.path.exists(path) and os.path.getsize(path) > 0)
    with open(path, "a") as fh:
        if need_header:
            fh.write(header + "\n")
        fh.write(row + "\n")


# ------------------------------------------------------------------- 2D -----
@dataclass
class Tensor2:
    k_xx: float
    k_yx: float
    k_xy: float
    k_yy: float
    k_off: float
    recip: float
    k1: float
    k2: float
    km: float
    aniso: float
    theta: float
    alpha_x: float
    alpha_y: float


def assemble2(rx, ry, mu, F) -> Tensor2:
    """LMB2d/main.cpp:326-353."""
    with np.errstate(divide="ignore", invalid="ignore"):
        k_xx, k_yx, k_xy, k_yy = (float(np.float64(mu) * v / np.float64(F))
                                  for v in (rx.q[0], rx.q[1], ry.q[0], ry.q[1]))
    k_off = 0.5 * (k_xy + k_yx)
    trace = k_xx + k_yy
    recip = abs(k_xy - k_yx) / abs(trace) if trace != 0.0 else math.nan
    km = 0.5 * (k_xx + k_yy)
    d1 = 0.5 * (k_xx - k_yy)
    d2 = k_off
    r = math.sqrt(d1 * d1 + d2 * d2)
    k1, k2 = km + r, km - r
    aniso = r / km if km != 0.0 else math.nan
    theta = 0.5 * math.atan2(d2, d1) * 180.0 / math.pi
    alpha_x = math.atan2(rx.q[1], rx.q[0]) * 180.0 / math.pi
    alpha_y = math.atan2(ry.q[1], ry.q[0]) * 180.0 / math.pi - 90.0
    return Tensor2(k_xx, k_yx, k_xy, k_yy, k_off, recip, k1, k2, km, aniso, theta, alpha_x, alpha_y)


def header2() -> str:
    return ("filename,ff,force,mu,porosity,"
            "steps_fx,conv_fx,steps_fy,conv_fy,"
            "qx_fx,qy_fx,qx_fy,qy_fy,"
            "se_qx_fx,se_qy_fx,se_qx_fy,se_qy_fy,"
            "k_xx,k_yx,k_xy,k_yy,k_off,recip_resid,"
            "k1,k2,k_mean,anisotropy,theta_deg,alpha_x_deg,alpha_y_deg,"
            "fieldres_fx,fieldres_fy")


def row2(filename, ff, F, mu, porosity, rx, ry, T: Tensor2) -> str:
    """LMB2d/main.cpp:396-405."""
    vals = [filename, fmt(ff), fmt(F), fmt(mu), fmt(porosity),
            fmt(rx.steps), fmt(rx.converged), fmt(ry.steps), fmt(ry.converged),
            fmt(rx.q[0]), fmt(rx.q[1]), fmt(ry.q[0]), fmt(ry.q[1]),
            fmt(rx.se[0]), fmt(rx.se[1]), fmt(ry.se[0]), fmt(ry.se[1]),
            fmt(T.k_xx), fmt(T.k_yx), fmt(T.k_xy), fmt(T.k_yy), fmt(T.k_off), fmt(T.recip),
            fmt(T.k1), fmt(T.k2), fmt(T.km), fmt(T.aniso), fmt(T.theta), fmt(T.alpha_x),
            fmt(T.alpha_y), fmt(rx.fieldres), fmt(ry.fieldres)]
    return ",".join(str(v) for v in vals)
