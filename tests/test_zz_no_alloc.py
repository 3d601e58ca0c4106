"""lbm_solve2d_noalloc: the D2Q9 solve on the library's static device scratch
(no device allocation inside the call), called through the C ABI and compared
with lbm_solve2d on the same inputs.

The file name sorts last so that, in a full run, these tests also run after
every other GPU test of the session (with the allocator pools of the earlier
tests warm); run alone, they pass in a fresh process as well.
"""
import ctypes as C
import ctypes.util
import re
from pathlib import Path

import numpy as np
import pytest

from flow_anizotropy_b200 import _lib
from flow_anizotropy_b200 import solver as S

ROOT = Path(__file__).resolve().parent.parent
SRC = ROOT / "flow_anizotropy_b200" / "csrc" / "engine2_noalloc.cu"

# Same kernels over the same work list in the same order as lbm_solve2d, so
# every number is expected bit for bit: the tolerance is zero.
TOL = 0.0

PRM = dict(eps=1e-3, lag=500, hold=3, min_steps=1000, max_steps=4000, avg_steps=500, avg_sample=50)
F = 2.5e-7
FORCES = [[F, 0.0], [0.0, F]]


def _solid(shape, seed, frac):
    s = (np.random.default_rng(seed).random(shape) < frac).astype(np.uint8)
    s.flat[0] = 0
    return s


def _call(ctx, entry, solid, forces=FORCES, prm=PRM, solid_ptr=None):
    ny, nx = solid.shape
    Fv = np.ascontiguousarray(np.asarray(forces, np.float64).reshape(-1, 2))
    ndir = Fv.shape[0]
    res = (_lib.Result2D * ndir)()
    vel = np.full((ndir, ny, nx, 2), np.nan, np.float32)
    P = S.Params2D(**prm).to_c()
    ptr = solid_ptr if solid_ptr is not None else solid.ctypes.data_as(C.POINTER(C.c_uint8))
    rc = getattr(ctx.L, entry)(ctx.h, ptr, nx, ny, ndir, Fv.ctypes.data_as(C.POINTER(C.c_double)),
                               C.byref(P), res, vel.ctypes.data_as(C.POINTER(C.c_float)))
    runs = [dict(q=np.array(r.q[:]), se=np.array(r.se[:]), steps=r.steps, converged=r.converged,
                 status=r.status, fieldres=r.fieldres) for r in res]
    return rc, runs, vel


def _assert_same(got, ref):
    rc_g, runs_g, vel_g = got
    rc_r, runs_r, vel_r = ref
    assert rc_g == rc_r
    assert rc_r in (_lib.LBM_OK, _lib.LBM_NOT_CONVERGED)
    for g, r in zip(runs_g, runs_r):
        assert (g["steps"], g["converged"], g["status"]) == (r["steps"], r["converged"], r["status"])
        np.testing.assert_allclose(g["q"], r["q"], rtol=TOL, atol=0)
        np.testing.assert_allclose(g["se"], r["se"], rtol=TOL, atol=0)
        np.testing.assert_allclose(g["fieldres"], r["fieldres"], rtol=TOL, atol=0)
    np.testing.assert_allclose(vel_g, vel_r, rtol=TOL, atol=0)


def test_source_allocates_nothing():
    """The entry point's translation unit calls no allocator (comments aside)."""
    code = SRC.read_text()
    code = re.sub(r"/\*.*?\*/", "", code, flags=re.S)
    code = re.sub(r"//[^\n]*", "", code)
    for bad in ("cudaMalloc", "cudaFree", "cudaHostAlloc", "DevMem", "malloc(", "new ",
                "std::vector", "torch"):
        assert bad not in code, bad
    assert re.search(r"static\s+__device__\s+__align__\(256\)\s+unsigned char\s+g_scratch2d\[", code)
    assert "cudaGetSymbolAddress" in code


@pytest.mark.gpu
def test_two_calls_match_solve2d(gpu):
    solid = _solid((64, 64), 3, 0.25)
    ref = _call(gpu, "lbm_solve2d", solid)
    first = _call(gpu, "lbm_solve2d_noalloc", solid)
    second = _call(gpu, "lbm_solve2d_noalloc", solid)
    _assert_same(first, ref)
    _assert_same(second, ref)


@pytest.mark.gpu
def test_full_cell_then_ragged_cell(gpu):
    """The largest accepted cell, then a smaller ragged one in the same scratch
    (left-over fields and controller state of the first call must not leak)."""
    big = _solid((256, 256), 11, 0.3)
    prm = dict(PRM, max_steps=2000)
    _assert_same(_call(gpu, "lbm_solve2d_noalloc", big, prm=prm), _call(gpu, "lbm_solve2d", big, prm=prm))
    small = _solid((40, 33), 5, 0.3)
    _assert_same(_call(gpu, "lbm_solve2d_noalloc", small, forces=[[F, 0.0]]),
                 _call(gpu, "lbm_solve2d", small, forces=[[F, 0.0]]))


@pytest.mark.gpu
def test_device_resident_mask(gpu):
    import torch
    solid = _solid((48, 80), 7, 0.3)
    dev = torch.from_numpy(solid).to("cuda:0")
    torch.cuda.synchronize()
    ptr = C.cast(C.c_void_p(dev.data_ptr()), C.POINTER(C.c_uint8))
    _assert_same(_call(gpu, "lbm_solve2d_noalloc", solid, solid_ptr=ptr), _call(gpu, "lbm_solve2d", solid))


@pytest.mark.gpu
def test_limits_rejected(gpu):
    over = np.zeros((257, 256), np.uint8)
    rc, _, _ = _call(gpu, "lbm_solve2d_noalloc", over)
    assert rc == _lib.LBM_EINPUT
    assert "LBM_NOALLOC2D_MAX_CELLS" in gpu.error()
    ok = _solid((16, 16), 1, 0.2)
    rc, _, _ = _call(gpu, "lbm_solve2d_noalloc", ok, forces=[[F, 0.0], [0.0, F], [F, F]])
    assert rc == _lib.LBM_EINPUT
    assert "LBM_NOALLOC2D_MAX_DIRS" in gpu.error()
    bad = ok.copy()
    bad[3, 3] = 7
    rc, _, _ = _call(gpu, "lbm_solve2d_noalloc", bad)
    assert rc == _lib.LBM_EINPUT and "non-binary" in gpu.error()
    # a rejected call leaves the scratch usable
    _assert_same(_call(gpu, "lbm_solve2d_noalloc", ok), _call(gpu, "lbm_solve2d", ok))


def _pool_bytes(device):
    """(reserved, used) bytes of the device's default stream-ordered pool, the
    pool the library's other entry points allocate from (driver API, so it is
    the same pool whichever CUDA runtime copy asked for it)."""
    cu = C.CDLL(ctypes.util.find_library("cuda") or "libcuda.so.1")
    dev = C.c_int()
    assert cu.cuDeviceGet(C.byref(dev), device) == 0
    pool = C.c_void_p()
    assert cu.cuDeviceGetDefaultMemPool(C.byref(pool), dev) == 0
    out = []
    for attr in (5, 7):     # CU_MEMPOOL_ATTR_RESERVED_MEM_CURRENT, CU_MEMPOOL_ATTR_USED_MEM_CURRENT
        v = C.c_uint64()
        assert cu.cuMemPoolGetAttribute(pool, attr, C.byref(v)) == 0
        out.append(v.value)
    return tuple(out)


@pytest.mark.gpu
def test_second_call_allocates_nothing(gpu):
    """After a first call (which may load the module and its static array),
    a second call changes neither the device's free memory nor the default
    pool's reserved or used bytes, and gives the same results."""
    import torch
    solid = _solid((96, 80), 13, 0.25)
    first = _call(gpu, "lbm_solve2d_noalloc", solid)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    pool0 = _pool_bytes(0)
    second = _call(gpu, "lbm_solve2d_noalloc", solid)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    pool1 = _pool_bytes(0)
    assert free1 == free0, (free0, free1)
    assert pool1 == pool0, (pool0, pool1)
    _assert_same(second, first)
