"""Per-step parity of the D3Q19 kernels with the CPU oracle (GPU tests).

After n steps the device lattice (AA layout, extracted in the reference's
canonical post-collision form) must equal the oracle's f0:
  * FP64: bit for bit (same operation order, no FMA contraction on either side);
  * FP32 / FP16 / BF16 shifted storage: within the storage precision.
Sizes are non-cubic and odd so that every periodic wrap and mask-word edge is hit.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

SHAPES = [(5, 6, 7), (9, 11, 33), (12, 14, 16), (8, 8, 64), (3, 4, 70)]


def _solid(shape, seed, frac=0.3):
    s = (np.random.default_rng(seed).random(shape) < frac).astype(np.uint8)
    s.flat[0] = 0
    return s


def _oracle_after(solid, force, n, tau=1.0):
    o = O.State3D(solid, tau)
    o.reset(force)
    o.step(n)
    return o.f(), o.u(), o.q()


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("nsteps", [1, 2, 3, 10])
def test_fp64_bitwise(gpu, shape, nsteps):
    from flow_anizotropy_b200.solver import debug_steps3d
    solid = _solid(shape, sum(shape) + nsteps)
    force = [1e-6, 2e-7, -3e-7]
    f, u, q = debug_steps3d(solid, force, nsteps, precision="fp64")
    fo, uo, qo = _oracle_after(solid, force, nsteps)
    pore = solid == 0
    assert np.array_equal(f[pore], fo[pore])
    np.testing.assert_allclose(q, qo, rtol=1e-13, atol=1e-25)
    np.testing.assert_allclose(u[pore], uo[pore].astype(np.float32), rtol=2e-6, atol=1e-12)
    assert np.all(u[~pore] == 0)


@pytest.mark.parametrize("tau", [0.8, 1.3])
def test_fp64_bitwise_tau(gpu, tau):
    from flow_anizotropy_b200.solver import debug_steps3d
    solid = _solid((9, 11, 33), 7)
    force = [0, 1e-6, 0]
    f, u, q = debug_steps3d(solid, force, 6, tau=tau, precision="fp64")
    fo, uo, qo = _oracle_after(solid, force, 6, tau)
    pore = solid == 0
    assert np.array_equal(f[pore], fo[pore])


@pytest.mark.parametrize("prec,tol", [("fp32", 2e-6), ("fp16", 2e-3), ("bf16", 1.6e-2)])
def test_shifted_storage(gpu, prec, tol):
    """Deviation f - w after a few steps, relative to its own magnitude."""
    from flow_anizotropy_b200.solver import debug_steps3d
    solid = _solid((12, 14, 16), 5)
    force = [1e-6, 0, 0]
    w = np.array([1/3] + [1/18] * 6 + [1/36] * 12)
    for n in (1, 2, 5):
        f, u, q = debug_steps3d(solid, force, n, precision=prec)
        fo, uo, qo = _oracle_after(solid, force, n)
        pore = solid == 0
        d = (f[pore] - w) - (fo[pore] - w)
        scale = np.abs(fo[pore] - w).max()
        assert np.abs(d).max() <= tol * scale, (prec, n, np.abs(d).max() / scale)
        np.testing.assert_allclose(q, qo, rtol=tol * 5)


@pytest.mark.parametrize("prec", ["fp64", "fp32", "fp16", "bf16"])
def test_every_variant_agrees(gpu, prec):
    """Each step-kernel variant (pore voxels per thread x register budget) gives
    the same populations and fluxes: bit for bit within a precision."""
    from flow_anizotropy_b200 import _lib
    from flow_anizotropy_b200.solver import debug_steps3d
    solid = _solid((10, 13, 37), 21)
    force = [3e-7, 1e-6, 0]
    nv = _lib.load().lbm_variant_count(_lib.PRECISIONS[prec])
    ref = None
    for v in range(nv):
        for n in (3, 4):
            f, u, q = debug_steps3d(solid, force, n, precision=prec, variant=v)
            if v == 0:
                ref = (ref or {})
                ref[n] = (f, q)
            else:
                assert np.array_equal(f, ref[n][0]), (prec, v, n)
                assert np.array_equal(q, ref[n][1]), (prec, v, n)   # fluxes summed in one order


@pytest.mark.parametrize("prec", ["fp32", "fp16", "bf16"])
def test_every_odd_variant_agrees_general_tau(gpu, prec):
    """tau != 1 (the general operator, packed and scalar forms): every odd
    variant with the same even kernel gives the same populations, bit for
    bit, after odd and even step counts."""
    from flow_anizotropy_b200 import _lib
    from flow_anizotropy_b200.solver import debug_steps3d
    solid = _solid((10, 13, 37), 23)
    force = [-4e-7, 2e-7, 1e-6]
    nv = _lib.load().lbm_variant_count(_lib.PRECISIONS[prec])
    nv_even = 15      # NVAR_EVEN_LP
    ref = {n: debug_steps3d(solid, force, n, tau=0.8, precision=prec, variant=1) for n in (3, 4)}
    assert nv == 5 * nv_even + 6 + 5 * nv_even
    for vo in range(1, 5):
        for n in (3, 4):
            f, u, q = debug_steps3d(solid, force, n, tau=0.8, precision=prec, variant=vo * nv_even + 1)
            assert np.array_equal(f, ref[n][0]) and np.array_equal(u, ref[n][1]), (prec, vo, n)
            assert np.array_equal(q, ref[n][2]), (prec, vo, n)
    # the pull-form variants (two lattices) after the 5 x 15 in-place ones,
    # then the two-lattice AA form of each odd variant with the same even one
    for v in list(range(5 * nv_even, 5 * nv_even + 6)) + [5 * nv_even + 6 + vo * nv_even + 1 for vo in range(5)]:
        for n in (3, 4):
            f, u, q = debug_steps3d(solid, force, n, tau=0.8, precision=prec, variant=v)
            assert np.array_equal(f, ref[n][0]) and np.array_equal(u, ref[n][1]), (prec, v, n)
            assert np.array_equal(q, ref[n][2]), (prec, v, n)


@pytest.mark.parametrize("prec,tol", [("fp32", 2e-6), ("fp16", 2e-3)])
def test_shifted_storage_general_tau(gpu, prec, tol):
    """tau != 1 takes the general (non-specialised) pair operator."""
    from flow_anizotropy_b200.solver import debug_steps3d
    solid = _solid((12, 14, 16), 9)
    force = [0, 0, 1e-6]
    w = np.array([1/3] + [1/18] * 6 + [1/36] * 12)
    for n in (1, 2, 5):
        f, u, q = debug_steps3d(solid, force, n, tau=0.8, precision=prec)
        fo, uo, qo = _oracle_after(solid, force, n, tau=0.8)
        pore = solid == 0
        d = (f[pore] - w) - (fo[pore] - w)
        scale = np.abs(fo[pore] - w).max()
        assert np.abs(d).max() <= tol * scale, (prec, n, np.abs(d).max() / scale)
