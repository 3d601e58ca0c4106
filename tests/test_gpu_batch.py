"""Batched solves (lbm_batch_*): many structures of uneven size resident
together, advanced by CUDA-graph chunks, retiring independently.  Every
result must equal the same solve run alone (the flux reduction sums tiles in
a fixed order, so alone and in the mix agree bit for bit), and admission must
respect the HBM budget."""
import numpy as np
import pytest

from flow_anizotropy_b200 import solver as S
from flow_anizotropy_b200 import structures as st

pytestmark = pytest.mark.gpu

PRM = dict(eps=1e-6, lag=100, hold=2, min_steps=200, max_steps=3000, avg_steps=50)


def _mix():
    out = []
    for i, (shape, r, phi) in enumerate([((16, 18, 20), 3.0, 0.6), ((24, 24, 24), 4.0, 0.5),
                                         ((12, 20, 33), 3.0, 0.55), ((20, 16, 16), 3.5, 0.65)]):
        out.append(st.sphere_packing(shape, r, phi, seed=40 + i, percolate=(True, True, True)))
    return out


def _forces(F=1e-6):
    return [[F, 0, 0], [0, F, 0], [0, 0, F]]


@pytest.mark.parametrize("prec", ["fp32", "fp64", "fp16"])
def test_batch_equals_alone(gpu, prec):
    structs = _mix()
    p = S.Params3D(precision=prec, **PRM)
    b = S.Batch(precision=prec, hbm_budget=4 * 2**30, chunk=32)
    for t, s in enumerate(structs):
        assert b.submit(s, _forces(), p, tag=t)
    done = {}
    for _ in range(1000):
        b.run(4)
        for tag, runs in b.poll():
            done[tag] = runs
        if len(done) == len(structs):
            break
    assert len(done) == len(structs) and b.active() == 0
    assert b.resident_bytes() == 0
    for t, s in enumerate(structs):
        alone, rc, _ = S.solve3d(s, _forces(), p)
        for a, m in zip(alone, done[t]):
            assert a.steps == m.steps and a.converged == m.converged
            assert np.array_equal(a.q, m.q), (prec, t, a.q, m.q)
            assert np.array_equal(a.se, m.se)


def test_batch_admission_and_continuous(gpu):
    """A budget that holds two structures: the third is refused until one
    retires, then admitted while the others keep running."""
    structs = _mix()[:3]
    p = S.Params3D(precision="fp32", **PRM)
    need = max(S.Batch.bytes_needed(s.shape, 3, "fp32") for s in structs)
    b = S.Batch(precision="fp32", hbm_budget=int(2.2 * need), chunk=16)
    assert b.submit(structs[0], _forces(), p, tag=0)
    assert b.submit(structs[1], _forces(), p, tag=1)
    admitted_late = b.submit(structs[2], _forces(), p, tag=2)
    done = {}
    for _ in range(2000):
        b.run(2)
        for tag, runs in b.poll():
            done[tag] = runs
        if not admitted_late:
            admitted_late = b.submit(structs[2], _forces(), p, tag=2)
        if len(done) == 3:
            break
    assert len(done) == 3
    alone, _, _ = S.solve3d(structs[2], _forces(), p)
    for a, m in zip(alone, done[2]):
        assert a.steps == m.steps and np.array_equal(a.q, m.q)


def test_batch_mixed_tau(gpu):
    """A solve with tau != 1 switches the batch to the general collision."""
    s = _mix()[0]
    p1 = S.Params3D(precision="fp32", **PRM)
    p8 = S.Params3D(precision="fp32", tau=0.8, **PRM)
    b = S.Batch(precision="fp32", hbm_budget=2**30, chunk=16)
    assert b.submit(s, _forces(), p1, tag=0)
    assert b.submit(s, _forces(), p8, tag=1)
    done = {}
    for _ in range(2000):
        b.run(4)
        done.update(dict(b.poll()))
        if len(done) == 2:
            break
    for tag, p in ((0, p1), (1, p8)):
        alone, _, _ = S.solve3d(s, _forces(), p)
        for a, m in zip(alone, done[tag]):
            assert a.steps == m.steps
            np.testing.assert_allclose(m.q, a.q, rtol=1e-6, atol=1e-20)


def test_batch_variant_choice(gpu):
    """lbm_batch_set_variant: any variant gives the default's bits; it is
    refused while solves are resident and for an unknown index."""
    from flow_anizotropy_b200 import _lib
    structs = _mix()[:2]
    p = S.Params3D(precision="fp16", **PRM)
    nve = 15                                    # even variants per odd variant
    pair_meta = 3 * nve + 1                     # odd: voxel pairs; even: neighbour records
    pull = 5 * nve                              # the two-lattice pull form, per direction
    aa2 = pull + 6                              # the two-lattice AA form of in-place variant v: aa2 + v
    out = {}
    # per direction (1, voxel pairs, pull forms, two-lattice AA) and grouped
    # even steps (6, 71 in place; -1 is the default 150, two-lattice AA)
    for v in (-1, 1, pair_meta, pull, pull + 3, aa2 + 4 * nve + 1, 6, 4 * nve + 11):
        b = S.Batch(precision="fp16", hbm_budget=4 * 2**30, chunk=32, variant=v)
        for t, s in enumerate(structs):
            assert b.submit(s, _forces(), p, tag=t)
        with pytest.raises(_lib.LBMError):
            b.ctx.check(b.ctx.L.lbm_batch_set_variant(b.h, 0))
        done = {}
        for _ in range(1000):
            b.run(4)
            for tag, runs in b.poll():
                done[tag] = runs
            if len(done) == len(structs):
                break
        out[v] = done
        b.close()
    for v in (1, pair_meta, pull, pull + 3, aa2 + 4 * nve + 1, 6, 4 * nve + 11):
        for t in range(len(structs)):
            for a, m in zip(out[-1][t], out[v][t]):
                assert a.steps == m.steps and np.array_equal(a.q, m.q) and np.array_equal(a.se, m.se), v
    b = S.Batch(precision="fp16", hbm_budget=4 * 2**30, chunk=32)
    with pytest.raises(_lib.LBMError):
        b.ctx.check(b.ctx.L.lbm_batch_set_variant(b.h, 10**6))
    # the grouped pull variants step every launch by structure; the batch
    # steps its odd launches per direction and refuses them
    with pytest.raises(_lib.LBMError, match="grouped"):
        b.ctx.check(b.ctx.L.lbm_batch_set_variant(b.h, pull + 4))
    with pytest.raises(_lib.LBMError, match="grouped"):
        b.ctx.check(b.ctx.L.lbm_batch_set_variant(b.h, pull + 5))
    b.close()


@pytest.mark.parametrize("prec", ["fp16", "fp32"])
def test_grouped_batch_slots_and_reuse(gpu, prec):
    """A grouped even-step variant in a batch (the 16-bit default; in-place
    variant 71 for FP32): structures of 4, 1 and 3 directions (groups of
    3 + 1, 1 and 3), directions finishing at different steps, a budget that
    makes later structures wait for a whole group to leave and reuse its
    slots: every result equals the solve alone bit for bit."""
    structs = _mix()
    F = 1e-6
    fsets = [_forces(F) + [[F / 3**0.5] * 3], [[0, F, 0]], _forces(F), [[F, 0, 0], [0, 0, F]]]
    p = S.Params3D(precision=prec, **PRM)
    v = -1 if prec == "fp16" else 4 * 15 + 11
    need = sum(S.Batch.bytes_needed(s.shape, len(f), prec) for s, f in zip(structs[:2], fsets[:2]))
    b = S.Batch(precision=prec, hbm_budget=int(1.05 * need), chunk=16, variant=v)
    pending = list(range(len(structs)))
    done = {}
    for _ in range(4000):
        while pending and b.submit(structs[pending[0]], fsets[pending[0]], p, tag=pending[0]):
            pending.pop(0)
        b.run(2)
        for tag, runs in b.poll():
            done[tag] = runs
        if len(done) == len(structs):
            break
    assert len(done) == len(structs) and not pending
    for t, s in enumerate(structs):
        alone, _, _ = S.solve3d(s, fsets[t], S.Params3D(precision=prec, variant=v, **PRM))
        assert len(done[t]) == len(alone)
        for a, m in zip(alone, done[t]):
            assert (a.steps, a.converged) == (m.steps, m.converged), t
            assert np.array_equal(a.q, m.q) and np.array_equal(a.se, m.se), t
