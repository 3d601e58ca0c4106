"""Python API of the B200 permeability solver (over liblbm's C ABI).

``solve3d`` / ``solve2d`` run any number of forcing directions of one
structure to convergence on the GPU; ``Batch`` keeps many structures resident
and advances them together (the continuous-batching engine the serving loop
uses).  Inputs may be numpy arrays (host) or CUDA torch tensors (device
buffers; their pointers are passed straight through).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import LBMError

FX_BASE = 2.5e-07      # body force at force factor 1 (LMB3d/lbm3d-perm.cpp:115, LMB2d/main.cpp:62)


def nu_of_tau(tau: float) -> float:
    """Kinematic viscosity cs^2 (tau - 1/2), rho0 = 1 (LMB3d/lbm3d-perm.cpp:114)."""
    return (1.0 / 3.0) * (tau - 0.5)


@dataclass
class Params3D:
    """Solver knobs; defaults are the reference's (LMB3d/lbm3d-perm.cpp:118-130)."""
    tau: float = 1.0
    eps: float = 1e-5
    lag: int = 2000
    hold: int = 2
    min_steps: int = 4000
    max_steps: int = 200000
    avg_steps: int = 2000
    precision: str = "fp64"
    criterion: str = "auto"     # "drift" (reference), "block", "batch", or auto: batch for fp16/bf16
    sample: int = 50            # block criteria: flux sampled every `sample` steps (gcd with lag if it does not divide it)
    ksigma: float = 3.0
    variant: int = _lib.LBM_VARIANT_DEFAULT   # or an index from tune3d

    def to_c(self) -> _lib.Params3D:
        prec = _lib.PRECISIONS[self.precision]
        crit = self.criterion
        if crit == "auto":
            crit = "batch" if prec in (_lib.FP16, _lib.BF16) else "drift"
        crit_code = {"drift": _lib.CRIT_DRIFT, "block": _lib.CRIT_BLOCK, "batch": _lib.CRIT_BATCH}[crit]
        return _lib.Params3D(tau=self.tau, eps=self.eps, lag=int(self.lag),
                             min_steps=int(self.min_steps), max_steps=int(self.max_steps),
                             avg_steps=int(self.avg_steps), hold=int(self.hold),
                             precision=prec, criterion=crit_code, variant=int(self.variant),
                             sample=_sample_for(int(self.lag), int(self.sample)), ksigma=float(self.ksigma))


def _sample_for(lag: int, sample: int) -> int:
    """The sample interval of the block criteria must divide lag: the largest
    common divisor of the two when `sample` does not."""
    if sample <= 0 or lag <= 0:
        return sample
    return sample if lag % sample == 0 else math.gcd(lag, sample)


@dataclass
class Result3D:
    q: np.ndarray
    se: np.ndarray
    steps: int
    converged: int
    status: int


@dataclass
class Params2D:
    """D2Q9 knobs; defaults are the reference's (LMB2d/main.cpp:64-79)."""
    tau: float = 1.0
    eps: float = 1e-3
    lag: int = 5000
    hold: int = 3
    min_steps: int = 10000
    max_steps: int = 500000
    avg_steps: int = 20000
    avg_sample: int = 50
    qfloor: float = 1e-2
    ksigma: float = 3.0

    def to_c(self) -> _lib.Params2D:
        return _lib.Params2D(tau=self.tau, eps=self.eps, lag=int(self.lag),
                             min_steps=int(self.min_steps), max_steps=int(self.max_steps),
                             avg_steps=int(self.avg_steps), avg_sample=int(self.avg_sample),
                             qfloor=self.qfloor, ksigma=self.ksigma, hold=int(self.hold),
                             reserved=0)


@dataclass
class Result2D:
    q: np.ndarray
    se: np.ndarray
    steps: int
    converged: int
    status: int
    fieldres: float


def _mask_ptr(solid, ndim):
    """(pointer, shape, keepalive) of a uint8 mask given as numpy or CUDA tensor."""
    if hasattr(solid, "data_ptr") and hasattr(solid, "is_cuda") and solid.is_cuda:
        if solid.dtype.__repr__() != "torch.uint8" or not solid.is_contiguous():
            raise ValueError("device mask must be a contiguous torch.uint8 tensor")
        if solid.dim() != ndim:
            raise ValueError(f"expected a {ndim}D mask")
        return C.cast(C.c_void_p(solid.data_ptr()), C.POINTER(C.c_uint8)), tuple(solid.shape), solid
    arr = np.ascontiguousarray(solid, dtype=np.uint8)
    if arr.ndim != ndim:
        raise ValueError(f"expected a {ndim}D mask, got shape {arr.shape}")
    return arr.ctypes.data_as(C.POINTER(C.c_uint8)), arr.shape, arr


def solve3d(solid, forces, params: Params3D | None = None, velocity: bool = False,
            device: int = 0):
    """Solve every forcing direction in ``forces`` (ndir x 3) on structure ``solid``.

    Returns (results, rc, vel) where rc is the ABI code (0 all converged,
    3 some not) and vel is ndir x nz x ny x nx x 3 float32 (or None).  Raises
    LBMError on bad input (code 2, the reference's exit 2) or CUDA errors.
    """
    params = params or Params3D()
    ctx = _lib.context(device)
    ptr, shape, keep = _mask_ptr(solid, 3)
    nz, ny, nx = shape
    F = np.ascontiguousarray(np.asarray(forces, dtype=np.float64).reshape(-1, 3))
    ndir = F.shape[0]
    res = (_lib.Result3D * ndir)()
    vel = np.zeros((ndir, nz, ny, nx, 3), np.float32) if velocity else None
    vp = vel.ctypes.data_as(C.POINTER(C.c_float)) if velocity else None
    P = params.to_c()
    rc = ctx.L.lbm_solve3d(ctx.h, ptr, nx, ny, nz, ndir,
                           F.ctypes.data_as(C.POINTER(C.c_double)), C.byref(P), res, vp)
    ctx.check(rc, ok=(_lib.LBM_OK, _lib.LBM_NOT_CONVERGED))
    del keep
    out = [Result3D(q=np.array(r.q[:]), se=np.array(r.se[:]), steps=int(r.steps),
                    converged=int(r.converged), status=int(r.status)) for r in res]
    return out, rc, vel


def solve2d(solid, forces, params: Params2D | None = None, velocity: bool = False,
            device: int = 0):
    """D2Q9 counterpart of solve3d; ``solid`` is [y, x], forces ndir x 2."""
    params = params or Params2D()
    ctx = _lib.context(device)
    ptr, shape, keep = _mask_ptr(solid, 2)
    ny, nx = shape
    F = np.ascontiguousarray(np.asarray(forces, dtype=np.float64).reshape(-1, 2))
    ndir = F.shape[0]
    res = (_lib.Result2D * ndir)()
    vel = np.zeros((ndir, ny, nx, 2), np.float32) if velocity else None
    vp = vel.ctypes.data_as(C.POINTER(C.c_float)) if velocity else None
    P = params.to_c()
    rc = ctx.L.lbm_solve2d(ctx.h, ptr, nx, ny, ndir,
                           F.ctypes.data_as(C.POINTER(C.c_double)), C.byref(P), res, vp)
    ctx.check(rc, ok=(_lib.LBM_OK, _lib.LBM_NOT_CONVERGED))
    del keep
    out = [Result2D(q=np.array(r.q[:]), se=np.array(r.se[:]), steps=int(r.steps),
                    converged=int(r.converged), status=int(r.status),
                    fieldres=float(r.fieldres)) for r in res]
    return out, rc, vel


def solve2d_many(solids, forces, params: Params2D | None = None, device: int = 0):
    """Several structures of one cell size (array [n, y, x]) along the same
    forcing directions in one launch per step; returns (runs [n][ndir], rc).
    Each structure's results equal solve2d of it alone."""
    params = params or Params2D()
    ctx = _lib.context(device)
    arr = np.ascontiguousarray(solids, dtype=np.uint8)
    n, ny, nx = arr.shape
    F = np.ascontiguousarray(np.asarray(forces, dtype=np.float64).reshape(-1, 2))
    ndir = F.shape[0]
    res = (_lib.Result2D * (n * ndir))()
    P = params.to_c()
    rc = ctx.L.lbm_solve2d_many(ctx.h, n, arr.ctypes.data_as(C.POINTER(C.c_uint8)), nx, ny, ndir,
                                F.ctypes.data_as(C.POINTER(C.c_double)), C.byref(P), res)
    ctx.check(rc, ok=(_lib.LBM_OK, _lib.LBM_NOT_CONVERGED))
    runs = [[Result2D(q=np.array(r.q[:]), se=np.array(r.se[:]), steps=int(r.steps), converged=int(r.converged),
                      status=int(r.status), fieldres=float(r.fieldres)) for r in res[k * ndir:(k + 1) * ndir]]
            for k in range(n)]
    return runs, rc


def debug_steps3d(solid, force, nsteps, tau=1.0, precision="fp64", variant=0, device=0):
    """Exactly ``nsteps`` steps; returns (f [z,y,x,19] float64, u [z,y,x,3] float32, q)."""
    ctx = _lib.context(device)
    arr = np.ascontiguousarray(solid, dtype=np.uint8)
    nz, ny, nx = arr.shape
    f = np.zeros((nz, ny, nx, 19), np.float64)
    u = np.zeros((nz, ny, nx, 3), np.float32)
    q = (C.c_double * 3)()
    Fv = (C.c_double * 3)(*[float(v) for v in force])
    rc = ctx.L.lbm_debug_steps3d(ctx.h, arr.ctypes.data_as(C.POINTER(C.c_uint8)), nx, ny, nz,
                                 Fv, float(tau), _lib.PRECISIONS[precision], int(variant),
                                 int(nsteps), f.ctypes.data_as(C.POINTER(C.c_double)),
                                 u.ctypes.data_as(C.POINTER(C.c_float)), q)
    ctx.check(rc)
    return f, u, np.array(q[:])


def debug_steps2d(solid, force, nsteps, tau=1.0, device=0):
    """Exactly ``nsteps`` D2Q9 steps; returns (f [y,x,9], u [y,x,2], q)."""
    ctx = _lib.context(device)
    arr = np.ascontiguousarray(solid, dtype=np.uint8)
    ny, nx = arr.shape
    f = np.zeros((ny, nx, 9), np.float32)
    u = np.zeros((ny, nx, 2), np.float32)
    q = (C.c_double * 2)()
    Fv = (C.c_double * 2)(*[float(v) for v in force])
    rc = ctx.L.lbm_debug_steps2d(ctx.h, arr.ctypes.data_as(C.POINTER(C.c_uint8)), nx, ny, Fv,
                                 float(tau), int(nsteps), f.ctypes.data_as(C.POINTER(C.c_float)),
                                 u.ctypes.data_as(C.POINTER(C.c_float)), q)
    ctx.check(rc)
    return f, u, np.array(q[:])


def variant_count(precision="fp32") -> int:
    """Number of step-kernel variants of a storage precision."""
    return int(_lib.load().lbm_variant_count(_lib.PRECISIONS[precision]))


def tune3d(solid, ndir=3, precision="fp32", nsteps=200, device=0):
    """Time every step-kernel variant on this structure; returns (best, ms_per_step list)."""
    ctx = _lib.context(device)
    arr = np.ascontiguousarray(solid, dtype=np.uint8)
    nz, ny, nx = arr.shape
    prec = _lib.PRECISIONS[precision]
    nv = ctx.L.lbm_variant_count(prec)
    ms = (C.c_double * nv)()
    best = C.c_int(0)
    ctx.check(ctx.L.lbm_tune3d(ctx.h, arr.ctypes.data_as(C.POINTER(C.c_uint8)), nx, ny, nz,
                               int(ndir), prec, int(nsteps), ms, C.byref(best)))
    return int(best.value), list(ms)


# --------------------------------------------------------------- batching ---
@dataclass
class _Pending:
    tag: int
    ndir: int
    results: dict = field(default_factory=dict)


class Batch:
    """Resident set of 3D solves advanced together (lbm_batch_* in include/lbm.h).

    ``submit`` admits a structure with its forcing directions if the HBM
    budget allows (returns False otherwise); ``run`` advances every resident
    solve by ``chunks`` CUDA-graph launches of ``chunk`` steps; ``poll``
    returns the structures whose every direction has finished.
    """

    def __init__(self, precision="fp16", hbm_budget=150 * 2**30, chunk=64, device=0,
                 variant=_lib.LBM_VARIANT_DEFAULT):
        self.ctx = _lib.context(device)
        self.precision = precision
        h = C.c_void_p()
        self.ctx.check(self.ctx.L.lbm_batch_create(self.ctx.h, C.byref(h),
                                                   _lib.PRECISIONS[precision],
                                                   int(hbm_budget), int(chunk)))
        self.h = h
        if variant != _lib.LBM_VARIANT_DEFAULT:
            self.ctx.check(self.ctx.L.lbm_batch_set_variant(h, int(variant)))
        self.chunk = chunk
        self._pending: dict[int, _Pending] = {}

    @staticmethod
    def bytes_needed(shape, ndir=3, precision="fp16") -> int:
        nz, ny, nx = shape
        return int(_lib.load().lbm_batch_bytes3d(nx, ny, nz, ndir, _lib.PRECISIONS[precision]))

    def submit(self, solid, forces, params: Params3D, tag: int) -> bool:
        ptr, shape, keep = _mask_ptr(solid, 3)
        nz, ny, nx = shape
        F = np.ascontiguousarray(np.asarray(forces, dtype=np.float64).reshape(-1, 3))
        P = params.to_c()
        rc = self.ctx.L.lbm_batch_submit3d(self.h, ptr, nx, ny, nz, F.shape[0],
                                           F.ctypes.data_as(C.POINTER(C.c_double)),
                                           C.byref(P), int(tag))
        del keep
        if rc == _lib.LBM_EBUSY:
            return False
        self.ctx.check(rc)
        self._pending[int(tag)] = _Pending(tag=int(tag), ndir=F.shape[0])
        return True

    def run(self, chunks: int = 1):
        self.ctx.check(self.ctx.L.lbm_batch_run(self.h, int(chunks)))

    def poll(self):
        """[(tag, [Result3D per direction])] for structures now complete."""
        done = []
        cap = 256
        tags = (C.c_longlong * cap)()
        dirs = (C.c_int * cap)()
        res = (_lib.Result3D * cap)()
        while True:
            n = C.c_int(0)
            self.ctx.check(self.ctx.L.lbm_batch_poll(self.h, tags, dirs, res, cap, C.byref(n)))
            for i in range(n.value):
                r = res[i]
                p = self._pending[int(tags[i])]
                p.results[int(dirs[i])] = Result3D(q=np.array(r.q[:]), se=np.array(r.se[:]),
                                                   steps=int(r.steps), converged=int(r.converged),
                                                   status=int(r.status))
                if len(p.results) == p.ndir:
                    done.append((p.tag, [p.results[j] for j in range(p.ndir)]))
                    del self._pending[p.tag]
            if n.value < cap:
                break
        return done

    def active(self) -> int:
        return int(self.ctx.L.lbm_batch_active(self.h))

    def resident_bytes(self) -> int:
        return int(self.ctx.L.lbm_batch_resident_bytes(self.h))

    def close(self):
        if getattr(self, "h", None):
            self.ctx.L.lbm_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


__all__ = ["Params3D", "Result3D", "Params2D", "Result2D", "solve3d", "solve2d", "Batch",
           "debug_steps3d", "debug_steps2d", "tune3d", "LBMError", "FX_BASE", "nu_of_tau"]
