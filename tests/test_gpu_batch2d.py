"""Several 2D structures per launch (lbm_solve2d_many) and the 2D dataset
driver built on it (flow_anizotropy_b200.batch2d): every structure's result
equals its solve alone, and the per-sample rows are byte-identical to the
lbm2d-perm drop-in's."""
from pathlib import Path

import numpy as np
import pandas as pd
import pytest

from flow_anizotropy_b200 import batch2d as B
from flow_anizotropy_b200 import cli2d
from flow_anizotropy_b200 import solver as S
from flow_anizotropy_b200.structure_io import save_dat

pytestmark = pytest.mark.gpu

PRM = dict(eps=1e-3, lag=500, hold=3, min_steps=1000, max_steps=4000, avg_steps=500, avg_sample=50)
EXTRA = "--size 48x40 --eps 1e-3 --lag 500 --hold 3 --min-steps 1000 --max-steps 4000 --avg-steps 500 --avg-sample 50"


def _solid(shape, seed, frac):
    s = (np.random.default_rng(seed).random(shape) < frac).astype(np.uint8)
    s.flat[0] = 0
    return s


def test_many_equals_alone(gpu):
    solids = np.stack([_solid((40, 48), 10 + k, 0.2 + 0.05 * k) for k in range(5)])
    F = 2.5e-7
    forces = [[F, 0.0], [0.0, F]]
    many, rc = S.solve2d_many(solids, forces, S.Params2D(**PRM))
    for k in range(len(solids)):
        alone, _, _ = S.solve2d(solids[k], forces, S.Params2D(**PRM))
        for a, m in zip(alone, many[k]):
            assert (a.steps, a.converged) == (m.steps, m.converged)
            assert np.array_equal(a.q, m.q) and np.array_equal(a.se, m.se) and a.fieldres == m.fieldres


def test_dataset_rows_equal_dropin(gpu, tmp_path):
    d = tmp_path / "ds"
    (d / "structures").mkdir(parents=True)
    rows = []
    for k in range(5):
        name = f"img{k}.dat"
        save_dat(d / "structures" / name, _solid((40, 48), 20 + k, 0.25))
        rows.append({"sample_id": k, "filename": name})
    pd.DataFrame(rows).to_csv(d / "structures.csv", index=False)
    res = B.run(str(d), ff=1.0, extra=EXTRA, group=3, log=lambda *a: None)
    assert res["solved"] == 5 and not res["failed"]
    for t in B.plan(str(d)):
        alone = tmp_path / f"alone{t.sample_id}.csv"
        rc = cli2d.run([t.structure, str(alone), "--quiet", "--ff", "1.0"] + EXTRA.split())
        assert rc in (0, 3)
        assert Path(t.out_csv).read_text() == alone.read_text(), t.sample_id
    again = B.run(str(d), ff=1.0, extra=EXTRA, group=3, log=lambda *a: None)
    assert again["solved"] == 0 and again["cached"] == 5
