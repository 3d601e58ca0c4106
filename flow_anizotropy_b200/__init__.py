"""B200-native lattice-Boltzmann permeability solver.

A drop-in for the D3Q19 / D2Q9 solvers of RafalTopolnicki/flow-anizotropy
(LMB3d/lbm3d-perm.cpp, LMB2d/lbm.cpp + LMB2d/main.cpp): same inputs (the
``.raw`` voxel file, 2D GIF/DAT), same CSV rows and exit codes, computed by
hand-written sm_100a CUDA kernels behind the C ABI in include/lbm.h.

    from flow_anizotropy_b200 import solve3d, Params3D
    runs, rc, _ = solve3d(solid, [[1e-6, 0, 0]], Params3D(precision="fp32"))
"""
from .solver import (Batch, LBMError, Params2D, Params3D, Result2D, Result3D,  # noqa: F401
                     solve2d, solve3d)

__version__ = "0.1.0"
