"""Build liblbm.so (the CUDA kernels and the C ABI) in-tree for sm_100a.

    python -m flow_anizotropy_b200.build

Each translation unit is compiled by nvcc with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3``; the FP64 D3Q19 and
the D2Q9 units additionally get ``-fmad=false`` so that their arithmetic keeps
the reference's rounding.  Objects go to ``flow_anizotropy_b200/_build/``,
the library to ``flow_anizotropy_b200/liblbm.so``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "liblbm.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
BASE = ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall"]
UNITS = {
    "k3d_f64.cu": ["-fmad=false"],
    "k2d.cu": ["-fmad=false"],
    "k3d_lp.cu": [],
    "k3d_m.cu": [],
    "k3d_md.cu": [],
    "k3d_reduce.cu": [],
    "engine.cu": [],
    "engine2.cu": [],
    "engine2_noalloc.cu": [],
    "engine_batch.cu": [],
    "gen3d.cu": ["-fmad=false"],
}


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    deps = [src] + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + [PKG.parent / "include" / "lbm.h"]
    t = obj.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def build(verbose: bool = False, force: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    cc = nvcc()
    jobs = []
    for name, extra in UNITS.items():
        src = CSRC / name
        obj = BUILD / (src.stem + ".o")
        if force or _stale(obj, src):
            cmd = [cc, *ARCH, *BASE, *extra, "-c", str(src), "-o", str(obj)]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            jobs.append(cmd)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        return r.stderr

    with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4) or 1) as pool:
        for log in pool.map(run, jobs):
            if verbose and log:
                print(log, file=sys.stderr)
    objs = [str(BUILD / (Path(n).stem + ".o")) for n in UNITS]
    if jobs or not LIB.exists() or force:
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [cc, *ARCH, "-shared", "-o", str(tmp), *objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
