"""ctypes wrapper over oracle/liboracle.so — TEST INFRASTRUCTURE ONLY.

The oracle is the C restatement of the reference solvers (LMB3d/lbm3d-perm.cpp,
LMB2d/lbm.cpp + LMB2d/main.cpp).  Only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg import this module, always as the checker; the
product (flow_anizotropy_b200 + liblbm.so) never does.

Also wraps the reference binaries built by oracle/build_ref.sh into
oracle/_ref/ (``ref_binary``), for tests that run the real reference.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
REF_DIR = HERE / "_ref"


class OR3DParams(C.Structure):
    _fields_ = [("tau", C.c_double), ("eps", C.c_double), ("lag", C.c_long),
                ("hold", C.c_int), ("min_steps", C.c_long), ("max_steps", C.c_long),
                ("avg_steps", C.c_long)]


class OR3DResult(C.Structure):
    _fields_ = [("q", C.c_double * 3), ("se", C.c_double * 3), ("steps", C.c_long),
                ("converged", C.c_int), ("status", C.c_int)]


class OR2DParams(C.Structure):
    _fields_ = [("tau", C.c_double), ("eps", C.c_double), ("lag", C.c_long),
                ("hold", C.c_int), ("min_steps", C.c_long), ("max_steps", C.c_long),
                ("avg_steps", C.c_long), ("avg_sample", C.c_long),
                ("qfloor", C.c_double), ("ksigma", C.c_double)]


class OR2DResult(C.Structure):
    _fields_ = [("q", C.c_double * 2), ("se", C.c_double * 2), ("steps", C.c_long),
                ("converged", C.c_int), ("status", C.c_int), ("fieldres", C.c_double)]


_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        vp, u8p = C.c_void_p, C.POINTER(C.c_uint8)
        L.or3d_new.restype = vp
        L.or3d_new.argtypes = [u8p, C.c_int, C.c_int, C.c_int, C.c_double]
        L.or3d_free.argtypes = [vp]
        L.or3d_reset.argtypes = [vp, C.c_double, C.c_double, C.c_double]
        L.or3d_step.argtypes = [vp]
        L.or3d_volumeavg.argtypes = [vp, C.POINTER(C.c_double)]
        L.or3d_f.restype = C.POINTER(C.c_double)
        L.or3d_f.argtypes = [vp]
        L.or3d_velocity.argtypes = [vp, C.POINTER(C.c_double)]
        L.or3d_solve.restype = C.c_int
        L.or3d_solve.argtypes = [u8p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double),
                                 C.POINTER(OR3DParams), C.POINTER(OR3DResult),
                                 C.POINTER(C.c_float)]
        L.or2d_new.restype = vp
        L.or2d_new.argtypes = [u8p, C.c_int, C.c_int, C.c_float]
        L.or2d_free.argtypes = [vp]
        L.or2d_reset.argtypes = [vp, C.c_float, C.c_float]
        L.or2d_step.argtypes = [vp]
        L.or2d_volumeavg.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.or2d_f.argtypes = [vp, C.POINTER(C.c_float)]
        L.or2d_velocity.argtypes = [vp, C.POINTER(C.c_float)]
        L.or2d_solve.restype = C.c_int
        L.or2d_solve.argtypes = [u8p, C.c_int, C.c_int, C.POINTER(C.c_double),
                                 C.POINTER(OR2DParams), C.POINTER(OR2DResult),
                                 C.POINTER(C.c_float)]
        _lib = L
    return _lib


def _u8(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint8))


# ---------------------------------------------------------------- 3D --------
DEF3D = dict(tau=1.0, eps=1e-5, lag=2000, hold=2, min_steps=4000, max_steps=200000,
             avg_steps=2000)


def solve3d(solid, force, velocity=False, **params):
    """One forcing direction of LMB3d/lbm3d-perm.cpp:solve().  solid is [z,y,x] uint8."""
    solid = np.ascontiguousarray(solid, dtype=np.uint8)
    nz, ny, nx = solid.shape
    p = dict(DEF3D, **params)
    P = OR3DParams(**p)
    R = OR3DResult()
    f = (C.c_double * 3)(*force)
    vel = np.zeros((nz, ny, nx, 3), np.float32) if velocity else None
    rc = lib().or3d_solve(_u8(solid), nx, ny, nz, f, C.byref(P), C.byref(R),
                          vel.ctypes.data_as(C.POINTER(C.c_float)) if velocity else None)
    out = dict(q=np.array(R.q[:]), se=np.array(R.se[:]), steps=int(R.steps),
               converged=int(R.converged), status=int(R.status), rc=rc)
    if velocity:
        out["vel"] = vel
    return out


class State3D:
    """Step-level access to the 3D oracle, for per-step parity checks."""

    def __init__(self, solid, tau=1.0):
        self.solid = np.ascontiguousarray(solid, dtype=np.uint8)
        self.nz, self.ny, self.nx = self.solid.shape
        self.n = self.solid.size
        self.h = lib().or3d_new(_u8(self.solid), self.nx, self.ny, self.nz, tau)

    def reset(self, force):
        lib().or3d_reset(self.h, *[float(v) for v in force])

    def step(self, n=1):
        for _ in range(n):
            lib().or3d_step(self.h)

    def q(self):
        q = (C.c_double * 3)()
        lib().or3d_volumeavg(self.h, q)
        return np.array(q[:])

    def f(self):
        """Post-collision distributions of the last step, [z,y,x,19]."""
        p = lib().or3d_f(self.h)
        a = np.ctypeslib.as_array(p, shape=(self.n * 19,)).copy()
        return a.reshape(self.nz, self.ny, self.nx, 19)

    def u(self):
        out = np.zeros(self.n * 3)
        lib().or3d_velocity(self.h, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out.reshape(self.nz, self.ny, self.nx, 3)

    def __del__(self):
        try:
            lib().or3d_free(self.h)
        except Exception:
            pass


# ---------------------------------------------------------------- 2D --------
DEF2D = dict(tau=1.0, eps=1e-3, lag=5000, hold=3, min_steps=10000, max_steps=500000,
             avg_steps=20000, avg_sample=50, qfloor=1e-2, ksigma=3.0)


def solve2d(solid, force, velocity=False, **params):
    """One forcing direction of LMB2d/main.cpp:solve().  solid is [y,x] uint8."""
    solid = np.ascontiguousarray(solid, dtype=np.uint8)
    ny, nx = solid.shape
    P = OR2DParams(**dict(DEF2D, **params))
    R = OR2DResult()
    f = (C.c_double * 2)(*force)
    vel = np.zeros((ny, nx, 2), np.float32) if velocity else None
    rc = lib().or2d_solve(_u8(solid), nx, ny, f, C.byref(P), C.byref(R),
                          vel.ctypes.data_as(C.POINTER(C.c_float)) if velocity else None)
    out = dict(q=np.array(R.q[:]), se=np.array(R.se[:]), steps=int(R.steps),
               converged=int(R.converged), status=int(R.status),
               fieldres=float(R.fieldres), rc=rc)
    if velocity:
        out["vel"] = vel
    return out


class State2D:
    def __init__(self, solid, tau=1.0):
        self.solid = np.ascontiguousarray(solid, dtype=np.uint8)
        self.ny, self.nx = self.solid.shape
        self.h = lib().or2d_new(_u8(self.solid), self.nx, self.ny, tau)

    def reset(self, force):
        lib().or2d_reset(self.h, float(force[0]), float(force[1]))

    def step(self, n=1):
        for _ in range(n):
            lib().or2d_step(self.h)

    def q(self):
        a, b = C.c_double(), C.c_double()
        lib().or2d_volumeavg(self.h, C.byref(a), C.byref(b))
        return np.array([a.value, b.value])

    def f(self):
        out = np.zeros(self.nx * self.ny * 9, np.float32)
        lib().or2d_f(self.h, out.ctypes.data_as(C.POINTER(C.c_float)))
        return out.reshape(self.ny, self.nx, 9)

    def u(self):
        out = np.zeros(self.nx * self.ny * 2, np.float32)
        lib().or2d_velocity(self.h, out.ctypes.data_as(C.POINTER(C.c_float)))
        return out.reshape(self.ny, self.nx, 2)

    def __del__(self):
        try:
            lib().or2d_free(self.h)
        except Exception:
            pass


# ------------------------------------------------------- reference binaries --
def ref_binary(name: str) -> Path | None:
    """Path of a reference binary built by oracle/build_ref.sh, or None."""
    p = REF_DIR / name
    return p if p.exists() and os.access(p, os.X_OK) else None
