"""The structure generator's CPU restatement (oracle/gen3d_oracle.py, with the
host-side sampling of flow_anizotropy_b200.gen3d) against the fixtures the
REFERENCE generator wrote (tests/golden/make_golden_gen3d.py): the same
draws, attempt counts, file names, thresholds and structure bytes, and the
same samples given up."""
import json
from pathlib import Path

import numpy as np
import pytest

from flow_anizotropy_b200.structure_io3d import load_structure
from oracle import gen3d_oracle as GO

GOLD = Path(__file__).resolve().parent / "golden" / "gen3d"
FIX = json.loads((GOLD / "rows.json").read_text())


def _cfg(r):
    return dict(seed=r["seed"], por_min=r["por_min"], por_max=r["por_max"], max_attempts=r["max_attempts"])


@pytest.mark.parametrize("r", FIX["rows"], ids=lambda r: f"seed{r['seed']}-s{r['sample_id']}-{r['max_attempts']}")
def test_oracle_reproduces_reference_generator(r):
    got = GO.sample(r["sample_id"], FIX["size"], **_cfg(r))
    if not r["kept"]:
        assert got is None
        return
    solid, row = got
    for k in ("filename", "n_modes", "attempts"):
        assert row[k] == r[k], k
    for k in ("aniso_A", "aniso_B", "k0", "porosity", "porosity_target", "threshold"):
        assert row[k] == r[k], k
    ref = load_structure(GOLD / r["filename"])
    assert np.array_equal(solid.astype(np.uint8), ref)


def test_oracle_percolation_axes():
    """An x-directed channel percolates in x only; an empty cell in every axis."""
    solid = np.ones((6, 7, 8), bool)
    solid[3, 4, :] = False
    assert GO.percolates(solid) == (True, False, False)
    assert GO.percolates(np.zeros((4, 4, 4), bool)) == (True, True, True)
    assert GO.percolates(np.ones((4, 4, 4), bool)) == (False, False, False)
