"""ctypes binding of liblbm.so (include/lbm.h).

The library is built in-tree (``python -m flow_anizotropy_b200.build``).
There is no fallback: if it is missing or fails to load, every solver entry
point raises, because the CUDA path is the only implementation.
"""
from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "liblbm.so"

LBM_OK, LBM_EINPUT, LBM_NOT_CONVERGED, LBM_EBUSY, LBM_ECUDA = 0, 2, 3, 4, -1
LBM_VARIANT_DEFAULT = -1      # the library's per-precision default step-kernel variant
FP64, FP32, FP16, BF16, M32, M64, MD32 = 0, 1, 2, 3, 4, 5, 6
PRECISIONS = {"fp64": FP64, "fp32": FP32, "fp16": FP16, "bf16": BF16, "m32": M32, "m64": M64,
              "md32": MD32}
CRIT_DRIFT, CRIT_BLOCK, CRIT_BATCH = 0, 1, 2

# Exported symbols, exactly those include/lbm.h declares.
SYMBOLS = (
    "lbm_version", "lbm_create", "lbm_destroy", "lbm_last_error", "lbm_stream",
    "lbm_solve3d", "lbm_solve2d", "lbm_solve2d_many", "lbm_solve2d_noalloc",
    "lbm_batch_create", "lbm_batch_set_variant", "lbm_batch_destroy", "lbm_batch_bytes3d", "lbm_batch_submit3d",
    "lbm_batch_run", "lbm_batch_poll", "lbm_batch_active", "lbm_batch_resident_bytes",
    "lbm_variant_count", "lbm_tune3d",
    "lbm_debug_steps3d", "lbm_debug_steps2d", "lbm_debug_bulk_wait",
    "lbm_trig_structure3d", "lbm_percolates3d",
)


class Params3D(C.Structure):
    _fields_ = [("tau", C.c_double), ("eps", C.c_double), ("lag", C.c_longlong),
                ("min_steps", C.c_longlong), ("max_steps", C.c_longlong),
                ("avg_steps", C.c_longlong), ("hold", C.c_int), ("precision", C.c_int),
                ("criterion", C.c_int), ("variant", C.c_int), ("sample", C.c_longlong),
                ("ksigma", C.c_double)]


class Result3D(C.Structure):
    _fields_ = [("q", C.c_double * 3), ("se", C.c_double * 3), ("steps", C.c_longlong),
                ("converged", C.c_int), ("status", C.c_int)]


class Params2D(C.Structure):
    _fields_ = [("tau", C.c_double), ("eps", C.c_double), ("lag", C.c_longlong),
                ("min_steps", C.c_longlong), ("max_steps", C.c_longlong),
                ("avg_steps", C.c_longlong), ("avg_sample", C.c_longlong),
                ("qfloor", C.c_double), ("ksigma", C.c_double), ("hold", C.c_int),
                ("reserved", C.c_int)]


class Result2D(C.Structure):
    _fields_ = [("q", C.c_double * 2), ("se", C.c_double * 2), ("steps", C.c_longlong),
                ("converged", C.c_int), ("status", C.c_int), ("fieldres", C.c_double)]


class LBMError(RuntimeError):
    """A liblbm call failed; ``code`` is the ABI return code."""

    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


_lib = None
_lock = threading.Lock()


def load(path: Path | str | None = None):
    """Load liblbm.so and declare every prototype.  Raises if it is absent."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        p = Path(path) if path else LIB_PATH
        if not p.exists():
            raise RuntimeError(
                f"{p} is missing: build the CUDA library first "
                "(python -m flow_anizotropy_b200.build); there is no CPU fallback")
        L = C.CDLL(str(p))
        vp, u8p, dp, fp = C.c_void_p, C.POINTER(C.c_uint8), C.POINTER(C.c_double), C.POINTER(C.c_float)
        L.lbm_version.restype = C.c_int
        L.lbm_create.argtypes = [C.POINTER(vp), C.c_int]
        L.lbm_create.restype = C.c_int
        L.lbm_destroy.argtypes = [vp]
        L.lbm_destroy.restype = None
        L.lbm_last_error.argtypes = [vp]
        L.lbm_last_error.restype = C.c_char_p
        L.lbm_stream.argtypes = [vp]
        L.lbm_stream.restype = C.c_void_p
        L.lbm_solve3d.argtypes = [vp, u8p, C.c_int, C.c_int, C.c_int, C.c_int, dp,
                                  C.POINTER(Params3D), C.POINTER(Result3D), fp]
        L.lbm_solve3d.restype = C.c_int
        L.lbm_solve2d.argtypes = [vp, u8p, C.c_int, C.c_int, C.c_int, dp,
                                  C.POINTER(Params2D), C.POINTER(Result2D), fp]
        L.lbm_solve2d.restype = C.c_int
        L.lbm_solve2d_many.argtypes = [vp, C.c_int, u8p, C.c_int, C.c_int, C.c_int, dp,
                                       C.POINTER(Params2D), C.POINTER(Result2D)]
        L.lbm_solve2d_many.restype = C.c_int
        L.lbm_solve2d_noalloc.argtypes = L.lbm_solve2d.argtypes
        L.lbm_solve2d_noalloc.restype = C.c_int
        L.lbm_batch_create.argtypes = [vp, C.POINTER(vp), C.c_int, C.c_longlong, C.c_int]
        L.lbm_batch_create.restype = C.c_int
        L.lbm_batch_set_variant.argtypes = [vp, C.c_int]
        L.lbm_batch_set_variant.restype = C.c_int
        L.lbm_batch_destroy.argtypes = [vp]
        L.lbm_batch_destroy.restype = None
        L.lbm_batch_bytes3d.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
        L.lbm_batch_bytes3d.restype = C.c_longlong
        L.lbm_batch_submit3d.argtypes = [vp, u8p, C.c_int, C.c_int, C.c_int, C.c_int, dp,
                                         C.POINTER(Params3D), C.c_longlong]
        L.lbm_batch_submit3d.restype = C.c_int
        L.lbm_batch_run.argtypes = [vp, C.c_int]
        L.lbm_batch_run.restype = C.c_int
        L.lbm_batch_poll.argtypes = [vp, C.POINTER(C.c_longlong), C.POINTER(C.c_int),
                                     C.POINTER(Result3D), C.c_int, C.POINTER(C.c_int)]
        L.lbm_batch_poll.restype = C.c_int
        L.lbm_batch_active.argtypes = [vp]
        L.lbm_batch_active.restype = C.c_int
        L.lbm_batch_resident_bytes.argtypes = [vp]
        L.lbm_batch_resident_bytes.restype = C.c_longlong
        L.lbm_variant_count.argtypes = [C.c_int]
        L.lbm_variant_count.restype = C.c_int
        L.lbm_tune3d.argtypes = [vp, u8p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                 dp, C.POINTER(C.c_int)]
        L.lbm_tune3d.restype = C.c_int
        L.lbm_debug_bulk_wait.argtypes = [vp, C.c_ulonglong, C.c_int]
        L.lbm_debug_bulk_wait.restype = C.c_int
        L.lbm_debug_steps3d.argtypes = [vp, u8p, C.c_int, C.c_int, C.c_int, dp, C.c_double,
                                        C.c_int, C.c_int, C.c_longlong, dp, fp, dp]
        L.lbm_debug_steps3d.restype = C.c_int
        L.lbm_debug_steps2d.argtypes = [vp, u8p, C.c_int, C.c_int, dp, C.c_double,
                                        C.c_longlong, fp, fp, dp]
        L.lbm_debug_steps2d.restype = C.c_int
        ip = C.POINTER(C.c_int32)
        L.lbm_trig_structure3d.argtypes = [vp, C.c_int, C.c_int, ip, dp, dp, C.c_double, C.c_double, u8p, dp]
        L.lbm_trig_structure3d.restype = C.c_int
        L.lbm_percolates3d.argtypes = [vp, u8p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int)]
        L.lbm_percolates3d.restype = C.c_int
        _lib = L
        return L


class Context:
    """One liblbm context (device + stream).  Not thread-safe; one per process is enough."""

    def __init__(self, device: int = 0):
        self.L = load()
        h = C.c_void_p()
        rc = self.L.lbm_create(C.byref(h), int(device))
        if rc != LBM_OK:
            raise LBMError(rc, "lbm_create failed: " + self.L.lbm_last_error(None).decode())
        self.h = h
        self.device = device

    @property
    def stream(self) -> int:
        """cudaStream_t of the context, as an integer (for torch.cuda.ExternalStream)."""
        return int(self.L.lbm_stream(self.h) or 0)

    def error(self) -> str:
        return self.L.lbm_last_error(self.h).decode()

    def check(self, rc: int, ok=(LBM_OK,)) -> int:
        if rc not in ok:
            raise LBMError(rc, self.error())
        return rc

    def close(self):
        if getattr(self, "h", None):
            self.L.lbm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_ctx: dict[int, Context] = {}


def context(device: int = 0) -> Context:
    """The process-wide context for a device."""
    if device not in _ctx:
        _ctx[device] = Context(device)
    return _ctx[device]
