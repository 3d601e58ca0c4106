"""Driver-side batching (flow_anizotropy_b200.batch3d) on the GPU: the
per-sample CSVs of a whole dataset solved through the resident batch are
byte-identical to the rows the lbm3d-perm drop-in writes for each structure
alone; a rerun solves nothing, an incomplete CSV is redone, and a bad
structure is reported without stopping the others."""
import os
from pathlib import Path

import numpy as np
import pytest

from flow_anizotropy_b200 import batch3d as B
from flow_anizotropy_b200 import cli3d
from flow_anizotropy_b200.structure_io3d import save_structure

from test_host import _dataset

pytestmark = pytest.mark.gpu

EXTRA = "--eps 1e-6 --lag 200 --hold 2 --min-steps 400 --max-steps 4000 --avg-steps 100"


@pytest.mark.parametrize("prec,validate", [("fp32", False), ("fp64", True)])
def test_dataset_rows_equal_dropin(gpu, tmp_path, prec, validate):
    d = _dataset(tmp_path, [(16, 18, 20), (20, 16, 18), (18, 20, 16), (16, 16, 16)], seed=3)
    extra = EXTRA + (" --validate" if validate else "")
    res = B.run(str(d), ff=2.0, extra=extra, precision=prec, chunk=64, log=lambda *a: None)
    assert res["solved"] == 4 and res["cached"] == 0 and not res["failed"]
    for t in B.plan(str(d)):
        alone = tmp_path / f"alone_{t.sample_id}.csv"
        rc = cli3d.run([t.structure, str(alone), "--quiet", "--ff", "2.0", "--precision", prec] + extra.split())
        assert rc in (0, 3)
        assert Path(t.out_csv).read_text() == alone.read_text(), t.sample_id
    # a rerun solves nothing; an incomplete file is redone to the same bytes
    again = B.run(str(d), ff=2.0, extra=extra, precision=prec, chunk=64, log=lambda *a: None)
    assert again["solved"] == 0 and again["cached"] == 4
    first = B.plan(str(d))[1]
    good = Path(first.out_csv).read_text()
    Path(first.out_csv).write_text(good.splitlines()[0] + "\n")
    redo = B.run(str(d), ff=2.0, extra=extra, precision=prec, chunk=64, log=lambda *a: None)
    assert redo["solved"] == 1 and redo["cached"] == 3
    assert Path(first.out_csv).read_text() == good


def test_bad_structure_is_reported(gpu, tmp_path):
    d = _dataset(tmp_path, [(16, 16, 16), (16, 16, 16)], seed=5)
    save_structure(d / "structures" / "s0001.raw", np.ones((16, 16, 16), np.uint8))   # all solid
    res = B.run(str(d), extra=EXTRA, precision="fp32", chunk=64, log=lambda *a: None)
    assert res["solved"] == 1 and [sid for sid, _ in res["failed"]] == [1]
    assert B.valid_result(B.plan(str(d))[0].out_csv)
    assert not os.path.exists(B.plan(str(d))[1].out_csv)
