"""The tau = 1 moment-projected form (LBM_M32 / LBM_M64 over the pore voxels,
LBM_MD32 over the dense box with TMA-staged planes) against the oracle.

It is the same operator and step sequence as the reference, holding (rho, u)
per pore voxel instead of 19 populations, so it must agree with the oracle to
roundoff: populations f* reconstructed from the moments per step, and whole
solves (same step counts, fluxes within 1e-8 for FP64 moments, 1e-4 FP32)."""
import numpy as np
import pytest

from flow_anizotropy_b200 import solver as S
from flow_anizotropy_b200 import structures as st
from oracle import oracle as O

pytestmark = pytest.mark.gpu
W = np.array([1/3] + [1/18] * 6 + [1/36] * 12)


def _solid(shape, seed, frac=0.3):
    s = (np.random.default_rng(seed).random(shape) < frac).astype(np.uint8)
    s.flat[0] = 0
    return s


@pytest.mark.parametrize("prec,tol", [("m64", 1e-9), ("m32", 3e-6), ("md32", 3e-6)])
@pytest.mark.parametrize("shape", [(5, 6, 7), (9, 11, 33), (3, 4, 70), (37, 17, 65), (1, 1, 40)])
def test_steps(gpu, prec, tol, shape):
    """Deviations f - w against the oracle's.  The oracle keeps O(1)
    populations, so its own rounding is ~ulp(1/3) = 5.6e-17 absolute: that,
    not the moments' precision, bounds the FP64 comparison (1e-9 of the
    ~1e-7 deviations)."""
    solid = _solid(shape, sum(shape))
    force = [1e-6, 2e-7, -3e-7]
    for n in (1, 2, 3, 10):
        f, u, q = S.debug_steps3d(solid, force, n, precision=prec)
        o = O.State3D(solid)
        o.reset(force)
        o.step(n)
        fo, uo, qo = o.f(), o.u(), o.q()
        pore = solid == 0
        d = (f[pore] - W) - (fo[pore] - W)
        assert np.abs(d).max() <= tol * np.abs(fo[pore] - W).max(), (prec, n)
        np.testing.assert_allclose(q, qo, rtol=tol * 10)
        assert np.all(u[~pore] == 0)


@pytest.mark.parametrize("shape", [(5, 6, 7), (37, 17, 65), (20, 9, 32)])
def test_dense_variants_agree(gpu, shape):
    """Every dense-form variant (z-segment length, ring depth) gives the same
    bits, and the dense form reproduces the compact FP32 moment form."""
    solid = _solid(shape, 7 + sum(shape))
    force = [1e-6, -2e-7, 3e-7]
    ref_f, ref_u, ref_q = S.debug_steps3d(solid, force, 6, precision="md32", variant=0)
    for v in range(1, S.variant_count("md32")):
        f, u, q = S.debug_steps3d(solid, force, 6, precision="md32", variant=v)
        assert np.array_equal(f, ref_f) and np.array_equal(u, ref_u) and np.array_equal(q, ref_q), v
    f, u, q = S.debug_steps3d(solid, force, 6, precision="m32")
    pore = solid == 0
    dev = np.abs(f[pore] - W).max()
    assert np.abs(f[pore] - ref_f[pore]).max() <= 1e-6 * dev
    np.testing.assert_allclose(q, ref_q, rtol=1e-6)


def test_moment_form_rejects_tau(gpu):
    with pytest.raises(S.LBMError) as e:
        S.solve3d(_solid((6, 6, 6), 1), [[1e-6, 0, 0]], S.Params3D(precision="m32", tau=0.8))
    assert e.value.code == 2 and "tau = 1" in str(e.value)


@pytest.mark.parametrize("prec,tol", [("m64", 1e-8), ("m32", 1e-4), ("md32", 1e-4)])
def test_solve_matches_oracle(gpu, prec, tol):
    solid = st.sphere_packing((20, 24, 28), 4.0, 0.6, seed=11, percolate=(True, True, True))
    F = 1e-6
    prm = dict(eps=1e-7, lag=200, hold=2, min_steps=400, max_steps=6000, avg_steps=100)
    forces = [[F, 0, 0], [0, F, 0], [0, 0, F]]
    runs, rc, vel = S.solve3d(solid, forces, S.Params3D(precision=prec, **prm), velocity=True)
    for j, f in enumerate(forces):
        r = O.solve3d(solid, f, velocity=(j == 0), **prm)
        g = runs[j]
        if prec == "m64":
            assert g.steps == r["steps"] and g.converged == r["converged"]
        scale = np.abs(r["q"]).max()
        assert np.abs(g.q - r["q"]).max() <= tol * scale, (prec, j)
        if j == 0:
            vmax = np.abs(r["vel"]).max()
            np.testing.assert_allclose(vel[0], r["vel"], rtol=1e-6 if prec == "m64" else 1e-4, atol=1e-6 * vmax)


@pytest.mark.parametrize("prec", ["m32", "md32"])
def test_batch_moments_equal_alone(gpu, prec):
    structs = [st.sphere_packing((16, 18, 20), 3.0, 0.6, seed=3, percolate=(True, True, True)),
               st.sphere_packing((24, 20, 22), 4.0, 0.5, seed=4, percolate=(True, True, True))]
    prm = dict(eps=1e-6, lag=100, hold=2, min_steps=200, max_steps=3000, avg_steps=50)
    p = S.Params3D(precision=prec, **prm)
    F = [[1e-6, 0, 0], [0, 1e-6, 0], [0, 0, 1e-6]]
    b = S.Batch(precision=prec, hbm_budget=2**30, chunk=32)
    for t, s in enumerate(structs):
        assert b.submit(s, F, p, tag=t)
    done = {}
    for _ in range(1000):
        b.run(4)
        done.update(dict(b.poll()))
        if len(done) == 2:
            break
    for t, s in enumerate(structs):
        alone, _, _ = S.solve3d(s, F, p)
        for a, m in zip(alone, done[t]):
            assert a.steps == m.steps and np.array_equal(a.q, m.q)
