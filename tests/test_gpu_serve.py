"""Serving with continuous batching: requests arriving while others run are
admitted between chunks, their work overlaps on the device, and each result
equals the same structure solved alone."""
import numpy as np
import pytest

from flow_anizotropy_b200 import solver as S
from flow_anizotropy_b200 import structures as st
from flow_anizotropy_b200.serve import Server

pytestmark = pytest.mark.gpu

PRM = dict(eps=1e-6, lag=100, hold=2, min_steps=200, max_steps=2500, avg_steps=50)
F = [[1e-6, 0, 0], [0, 1e-6, 0], [0, 0, 1e-6]]


@pytest.mark.parametrize("prec", ["fp32", "m32"])
def test_continuous_batching_matches_alone(gpu, prec):
    structs = [st.sphere_packing((14 + 2 * i, 16, 18), 3.0, 0.6, seed=60 + i, percolate=(True, True, True))
               for i in range(5)]
    p = S.Params3D(precision=prec, **PRM)
    srv = Server(precision=prec, hbm_budget=2**30, chunk=32)
    order = []
    # two requests up front, the rest arrive while those are running
    for s in structs[:2]:
        order.append(srv.submit(s, F, p))
    pumps = 0
    for s in structs[2:]:
        srv.pump(2)
        pumps += 1
        order.append(srv.submit(s, F, p))
    assert srv.stats.max_resident >= 2
    srv.drain(2)
    res = srv.results()
    assert len(res) == 5 and srv.stats.completed == 5
    assert all(lat >= 0 for lat in srv.stats.latencies)
    for rid, s in zip(order, structs):
        alone, _, _ = S.solve3d(s, F, p)
        for a, m in zip(alone, res[rid]):
            assert a.steps == m.steps and np.array_equal(a.q, m.q)
    srv.close()


def test_budget_queueing(gpu):
    s = st.sphere_packing((20, 20, 20), 3.0, 0.6, seed=70, percolate=(True, True, True))
    p = S.Params3D(precision="fp32", **PRM)
    probe = S.Batch(precision="fp32", hbm_budget=2**30, chunk=32)
    assert probe.submit(s, F, p, tag=0)
    need = probe.resident_bytes()            # exact admission charge of one request
    probe.close()
    assert 0 < need <= S.Batch.bytes_needed(s.shape, 3, "fp32")
    srv = Server(precision="fp32", hbm_budget=int(1.5 * need), chunk=32)
    ids = [srv.submit(s, F, p) for _ in range(3)]
    srv.pump(1)
    assert len(srv.inflight) == 1 and len(srv.queue) == 2      # one fits at a time
    srv.drain(4)
    assert sorted(srv.results()) == ids
    w = srv.stats.queue_waits
    assert w[0] <= w[1] <= w[2]
    srv.close()
