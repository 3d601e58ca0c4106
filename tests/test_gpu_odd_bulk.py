"""The bulk-staged odd step (odd variant 4: a shared-memory ring filled by
cp.async.bulk copies, persistent CTAs) against the pair kernel it restates
(odd variant 3): the populations, fluxes and whole solves must be identical
bit for bit.

The lattice here has more tiles than the persistent grid has CTAs times ring
buffers, so every CTA walks several work items and reuses its buffers; the
pore count is odd, so the last tile is partial and its last voxel's partner is
a padding slot.
"""
import numpy as np
import pytest

from flow_anizotropy_b200 import solver as S
from flow_anizotropy_b200 import structures as st

pytestmark = pytest.mark.gpu

NV_EVEN = 15          # even variants per odd variant (NVAR_EVEN_LP)
PAIR, BULK = 3, 4          # odd variant indices


def _variant(vo, ve=1):
    return vo * NV_EVEN + ve


def _solid(shape, seed, frac=0.38):
    s = (np.random.default_rng(seed).random(shape) < frac).astype(np.uint8)
    s.flat[0] = 0
    if int((s == 0).sum()) % 2 == 0:          # odd pore count: partial last pair
        s.flat[np.flatnonzero(s)[0]] = 0
    return s


@pytest.fixture(scope="module")
def big():
    s = _solid((100, 110, 120), 5)
    npore = int((s == 0).sum())
    assert npore % 2 == 1 and npore // 512 > 4 * 2 * 148      # > ring x persistent CTAs
    return s


@pytest.mark.parametrize("prec", ["fp32", "fp16", "bf16"])
def test_bulk_odd_step_equals_pair_kernel(gpu, big, prec):
    from flow_anizotropy_b200.solver import debug_steps3d
    force = [1e-6, -4e-7, 2e-7]
    for n in (1, 3, 4):
        f_p, u_p, q_p = debug_steps3d(big, force, n, precision=prec, variant=_variant(PAIR))
        f_b, u_b, q_b = debug_steps3d(big, force, n, precision=prec, variant=_variant(BULK))
        assert np.array_equal(f_b, f_p), (prec, n)
        assert np.array_equal(u_b, u_p), (prec, n)
        assert np.array_equal(q_b, q_p), (prec, n)


@pytest.mark.parametrize("prec", ["fp32", "fp16"])
def test_bulk_odd_whole_solves_identical(gpu, prec):
    """Three directions in one launch.  A solve that converges inside a
    64-step graph chunk leaves finished items in the chunk's remaining
    launches: the issuing thread's phase check skips them."""
    solid = st.sphere_packing((20, 24, 28), 4.0, 0.6, seed=11, percolate=(True, True, True))
    F = 1e-6
    forces = [[F, 0, 0], [0, F, 0], [0, 0, F]]
    prm = dict(eps=1e-7, lag=200, hold=2, min_steps=400, max_steps=6000, avg_steps=100)
    ref, rc0, vel0 = S.solve3d(solid, forces, S.Params3D(precision=prec, variant=_variant(PAIR), **prm),
                               velocity=True)
    got, rc, vel = S.solve3d(solid, forces, S.Params3D(precision=prec, variant=_variant(BULK), **prm),
                             velocity=True)
    assert rc == rc0
    for a, b in zip(ref, got):
        assert (a.steps, a.converged, a.status) == (b.steps, b.converged, b.status)
        assert np.array_equal(a.q, b.q) and np.array_equal(a.se, b.se)
    assert np.array_equal(vel, vel0)


def test_variant_table_has_bulk_odd(gpu):
    for prec in ("fp32", "fp16", "bf16"):
        assert S.variant_count(prec) == 5 * NV_EVEN + 6 + 5 * NV_EVEN   # + pull form + two-lattice AA form


def test_starved_waits_end_with_status(gpu):
    """Failure path of the bounded waits, with no fault: the producer issues
    nothing (test knob), the consumers' 2 ms waits run out, the solve ends
    with status 5 and the call fails with LBM_ECUDA; the context stays usable
    and the next solve is the normal one."""
    from flow_anizotropy_b200 import _lib
    solid = st.sphere_packing((20, 24, 28), 4.0, 0.6, seed=11, percolate=(True, True, True))
    F = 1e-6
    prm = dict(eps=1e-7, lag=200, hold=2, min_steps=400, max_steps=6000, avg_steps=100)
    p = S.Params3D(precision="fp16", variant=_variant(BULK), **prm)
    gpu.check(gpu.L.lbm_debug_bulk_wait(gpu.h, 2_000_000, 1))
    try:
        with pytest.raises(_lib.LBMError) as e:
            S.solve3d(solid, [[F, 0, 0]], p)
        assert e.value.code == _lib.LBM_ECUDA
        assert "gave up waiting" in gpu.error()
    finally:
        gpu.check(gpu.L.lbm_debug_bulk_wait(gpu.h, 0, 0))
    ok, rc, _ = S.solve3d(solid, [[F, 0, 0]], p)
    ref, rc0, _ = S.solve3d(solid, [[F, 0, 0]], S.Params3D(precision="fp16", variant=_variant(PAIR), **prm))
    assert rc == rc0 and ok[0].steps == ref[0].steps and np.array_equal(ok[0].q, ref[0].q)


@pytest.mark.parametrize("prec,default", [("fp32", 5 * NV_EVEN + 1), ("fp16", 5 * NV_EVEN + 6 + 4 * NV_EVEN + 9),
                                          ("bf16", 5 * NV_EVEN + 6 + 4 * NV_EVEN + 9),
                                          ("fp64", 0)])
def test_default_variant_is_the_tuned_pick_and_matches_variant_0(gpu, prec, default):
    """LBM_VARIANT_DEFAULT runs the listed variant; since every variant sums
    the fluxes in one order, a whole solve with it equals variant 0's bits."""
    solid = st.sphere_packing((20, 24, 28), 4.0, 0.6, seed=11, percolate=(True, True, True))
    F = 1e-6
    forces = [[F, 0, 0], [0, 0, F]]
    prm = dict(eps=1e-7, lag=200, hold=2, min_steps=400, max_steps=4000, avg_steps=100, precision=prec)
    runs = {}
    for v in (-1, default, 0):
        runs[v] = S.solve3d(solid, forces, S.Params3D(variant=v, **prm))[0]
    for v in (default, 0):
        for a, b in zip(runs[-1], runs[v]):
            assert (a.steps, a.converged) == (b.steps, b.converged)
            assert np.array_equal(a.q, b.q) and np.array_equal(a.se, b.se), (prec, v)
