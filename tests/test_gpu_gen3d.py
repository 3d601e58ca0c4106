"""Device structure generation (flow_anizotropy_b200.gen3d: lbm_trig_structure3d,
lbm_percolates3d) against the fixtures of the REFERENCE generator and the
CPU oracle: same attempts, file names and structure bytes; thresholds equal
to within the last bits of the field (the device cosine may differ from the
host's by an ulp); percolation identical to the tiled scipy labelling."""
import json
from pathlib import Path

import numpy as np
import pandas as pd
import pytest

from flow_anizotropy_b200 import batch3d as B
from flow_anizotropy_b200 import gen3d as G
from flow_anizotropy_b200.structure_io3d import load_structure
from oracle import gen3d_oracle as GO

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden" / "gen3d"
FIX = json.loads((GOLD / "rows.json").read_text())


def _cfg(r):
    return dict(seed=r["seed"], por_min=r["por_min"], por_max=r["por_max"], max_attempts=r["max_attempts"])


@pytest.mark.parametrize("r", FIX["rows"], ids=lambda r: f"seed{r['seed']}-s{r['sample_id']}-{r['max_attempts']}")
def test_device_generator_matches_reference(gpu, r):
    got = G.Generator(size=FIX["size"], **_cfg(r)).sample(r["sample_id"])
    if not r["kept"]:
        assert got is None
        return
    solid, row = got
    assert (row["filename"], row["n_modes"], row["attempts"]) == (r["filename"], r["n_modes"], r["attempts"])
    assert row["porosity_target"] == r["porosity_target"] and row["porosity"] == r["porosity"]
    assert abs(row["threshold"] - r["threshold"]) <= 1e-12 * max(1.0, abs(r["threshold"]))
    assert np.array_equal(solid.astype(np.uint8), load_structure(GOLD / r["filename"]))


@pytest.mark.parametrize("shape,frac,seed", [((5, 6, 7), 0.3, 1), ((9, 4, 13), 0.45, 2), ((1, 12, 12), 0.3, 3),
                                             ((16, 16, 16), 0.65, 4), ((24, 20, 18), 0.6, 5), ((3, 3, 40), 0.5, 6)])
def test_percolation_matches_oracle(gpu, shape, frac, seed):
    solid = np.random.default_rng(seed).random(shape) < frac
    gen = G.Generator(size=8)
    assert gen.percolates(solid.astype(np.uint8)) == GO.percolates(solid)


def test_dataset_feeds_batch_driver(gpu, tmp_path):
    """A generated dataset has the reference's layout and solves through batch3d."""
    out = tmp_path / "ds"
    rows = G.generate(str(out), 3, size=FIX["size"], log=lambda *a: None)
    df = pd.read_csv(out / "structures.csv")
    ref = [r for r in FIX["rows"] if r["seed"] == 0 and r["sample_id"] < 3]
    assert list(df.filename) == [r["filename"] for r in ref]
    assert len((out / "filelist.txt").read_text().splitlines()) == 3
    res = B.run(str(out), extra="--eps 1e-5 --lag 200 --min-steps 400 --max-steps 3000 --avg-steps 50",
                precision="fp32", chunk=64, log=lambda *a: None)
    assert res["solved"] == 3 and not res["failed"]
    assert len(rows) == 3
