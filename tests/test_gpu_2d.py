"""D2Q9 on the GPU against the 2D oracle: bit-identical populations per step,
and whole solves (block-mean controller) with identical step counts."""
import numpy as np
import pytest

from flow_anizotropy_b200 import solver as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _solid(shape, seed, frac=0.3):
    s = (np.random.default_rng(seed).random(shape) < frac).astype(np.uint8)
    s.flat[0] = 0
    return s


@pytest.mark.parametrize("shape", [(7, 9), (40, 33), (64, 64), (5, 100)])
@pytest.mark.parametrize("nsteps", [1, 2, 5, 20])
def test_bitwise_steps(gpu, shape, nsteps):
    solid = _solid(shape, nsteps + shape[0])
    force = [2.5e-7, -1e-7]
    f, u, q = S.debug_steps2d(solid, force, nsteps)
    o = O.State2D(solid)
    o.reset(force)
    o.step(nsteps)
    pore = solid == 0
    assert np.array_equal(f[pore], o.f()[pore])
    assert np.array_equal(u, o.u())
    np.testing.assert_allclose(q, o.q(), rtol=1e-14, atol=1e-30)


@pytest.mark.parametrize("prm", [
    dict(eps=1e-3, lag=500, hold=3, min_steps=1000, max_steps=4000, avg_steps=500, avg_sample=50),
    # lag and averaging lengths that are not multiples of the solve loop's
    # replayed chunk, so chunks and single launches interleave
    dict(eps=1e-3, lag=250, hold=3, min_steps=550, max_steps=3000, avg_steps=350, avg_sample=25),
])
def test_solve_matches_oracle(gpu, prm):
    solid = _solid((64, 64), 3, 0.25)
    F = 2.5e-7
    runs, rc, vel = S.solve2d(solid, [[F, 0], [0, F]], S.Params2D(**prm), velocity=True)
    for j, f in enumerate(([F, 0], [0, F])):
        r = O.solve2d(solid, f, velocity=True, **prm)
        g = runs[j]
        assert g.steps == r["steps"] and g.converged == r["converged"]
        np.testing.assert_allclose(g.q, r["q"], rtol=1e-12)
        np.testing.assert_allclose(g.se, r["se"], rtol=1e-6, atol=1e-20)
        assert abs(g.fieldres - r["fieldres"]) <= 1e-6 * max(abs(r["fieldres"]), 1e-30)
        assert np.array_equal(vel[j], r["vel"])
