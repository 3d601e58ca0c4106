"""Host-side logic without a GPU: structure I/O, CLI argument handling,
tensor algebra, generators, and the C ABI's exported symbols."""
import os
import re
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from flow_anizotropy_b200 import structures as st
from flow_anizotropy_b200 import tensor as T
from flow_anizotropy_b200.cli3d import parse, strtod, strtol, Die
from flow_anizotropy_b200.structure_io import load_dat, save_dat
from flow_anizotropy_b200.structure_io3d import (MAGIC_HEADER_BYTES, StructureError, load_structure,
                                                 porosity, read_raw_checked, save_structure)

ROOT = Path(__file__).resolve().parent.parent


def test_raw_roundtrip_non_cubic(tmp_path):
    # mirrors scripts/structure_io3d.py:75-127
    a = (np.random.default_rng(0).random((5, 7, 11)) > 0.5).astype(np.uint8)
    save_structure(tmp_path / "a.raw", a)
    b = load_structure(tmp_path / "a.raw")
    assert np.array_equal(a, b) and b.shape == (5, 7, 11)
    raw = (tmp_path / "a.raw").read_bytes()
    assert len(raw) == MAGIC_HEADER_BYTES + 5 * 7 * 11
    assert list(np.frombuffer(raw, "<i4", 3)) == [11, 7, 5]
    assert np.frombuffer(raw, np.uint8, offset=12)[(3 * 7 + 4) * 11 + 9] == a[3, 4, 9]
    assert abs(porosity(np.array([[[1, 0], [0, 0]]])) - 0.75) < 1e-12


@pytest.mark.parametrize("payload,msg", [
    (lambda a: a[:-3], "truncated payload"),
    (lambda a: a + b"\x00", "trailing bytes"),
    (lambda a: a[:8], "cannot read header"),
    (lambda a: np.array([0, 2, 2], "<i4").tobytes() + a[12:], "bad dimensions"),
])
def test_raw_checked_rejects(tmp_path, payload, msg):
    a = np.zeros((2, 3, 4), np.uint8)
    save_structure(tmp_path / "a.raw", a)
    (tmp_path / "b.raw").write_bytes(payload((tmp_path / "a.raw").read_bytes()))
    with pytest.raises(StructureError, match=msg):
        read_raw_checked(tmp_path / "b.raw")


def test_raw_checked_values(tmp_path):
    a = np.zeros((2, 3, 4), np.uint8)
    a[1, 1, 1] = 2
    (tmp_path / "a.raw").write_bytes(np.array([4, 3, 2], "<i4").tobytes() + a.tobytes())
    with pytest.raises(StructureError, match="non-binary voxel"):
        read_raw_checked(tmp_path / "a.raw")
    save_structure(tmp_path / "b.raw", np.ones((2, 2, 2), np.uint8))
    with pytest.raises(StructureError, match="no pore space"):
        read_raw_checked(tmp_path / "b.raw")
    with pytest.raises(StructureError, match="cannot open"):
        read_raw_checked(tmp_path / "missing.raw")


def test_dat_roundtrip(tmp_path):
    s = (np.random.default_rng(1).random((256, 256)) < 0.3).astype(np.uint8)
    save_dat(tmp_path / "s.dat", s)
    assert np.array_equal(load_dat(tmp_path / "s.dat"), s)


def test_strtol_strtod_match_c():
    assert strtol("12abc") == 12 and strtol("abc") == 0 and strtol("-7") == -7 and strtol(" 3") == 3
    assert strtod("1e-5x") == 1e-5 and strtod("x") == 0.0 and strtod("4") == 4.0


def test_cli3d_parse():
    s, r, cfg = parse(["a.raw", "b.csv", "--ff", "4", "--lag", "1000", "--eps", "1e-6", "--quiet",
                       "--validate", "--precision", "fp16"])
    assert (s, r) == ("a.raw", "b.csv")
    assert cfg["ff"] == 4.0 and cfg["lag"] == 1000 and cfg["eps"] == 1e-6 and cfg["quiet"] and cfg["validate"]
    with pytest.raises(Die, match="unknown option --bogus"):
        parse(["a.raw", "b.csv", "--bogus"])
    with pytest.raises(Die, match="missing value for --lag"):
        parse(["a.raw", "b.csv", "--lag"])
    for crit in ("drift", "block", "batch", "auto"):
        assert parse(["a.raw", "b.csv", "--criterion", crit])[2]["criterion"] == crit
    with pytest.raises(Die, match="unknown criterion"):
        parse(["a.raw", "b.csv", "--criterion", "median"])


def test_cli_exit_codes(tmp_path):
    # usage: 3D returns 2 on too few arguments, 2D returns 1 (LMB3d/lbm3d-perm.cpp:480, LMB2d/main.cpp:280)
    r3 = subprocess.run([sys.executable, "-m", "flow_anizotropy_b200.cli3d"], cwd=ROOT, capture_output=True)
    r2 = subprocess.run([sys.executable, "-m", "flow_anizotropy_b200.cli2d"], cwd=ROOT, capture_output=True)
    assert r3.returncode == 2 and r2.returncode == 1
    # input errors die with exit 2 and the solver's message, before any GPU work
    r = subprocess.run([str(ROOT / "flow_anizotropy_b200" / "bin" / "lbm3d-perm"), str(tmp_path / "x.raw"),
                        str(tmp_path / "o.csv")], capture_output=True, text=True)
    assert r.returncode == 2 and "lbm3d-perm: cannot open" in r.stderr
    assert not (tmp_path / "o.csv").exists()


def test_jacobi3_matches_numpy():
    rng = np.random.default_rng(3)
    for _ in range(50):
        M = rng.normal(size=(3, 3))
        A = M + M.T
        val, vec = T.jacobi3(A)
        w = np.sort(np.linalg.eigvalsh(A))[::-1]
        np.testing.assert_allclose(val, w, rtol=1e-10, atol=1e-12)
        V = np.array(vec)
        np.testing.assert_allclose(A @ V, V * np.array(val), atol=1e-10)


def test_fmt_like_cpp_stream():
    assert T.fmt(2.5e-07) == "2.5e-07" and T.fmt(4.0) == "4" and T.fmt(0.16666666666666666) == "0.1666666667"
    assert T.fmt(float("nan")) == "nan" and T.fmt(12) == "12" and T.fmt(1e-5) == "1e-05"


def test_generators_deterministic_and_on_target():
    a = st.sphere_packing(32, 4.0, 0.6, seed=5, percolate=(True, False, False))
    b = st.sphere_packing(32, 4.0, 0.6, seed=5, percolate=(True, False, False))
    assert np.array_equal(a, b)
    phi = 1 - a.mean()
    assert 0.55 < phi <= 0.60
    assert st.percolates(a)[0]


def test_percolation_slab():
    s = np.zeros((8, 8, 8), np.uint8)
    s[2] = 1                               # a full solid layer normal to z
    assert st.percolates(s) == (True, True, False)
    kept, ok = st.largest_spanning_cluster(s, "x")
    assert ok and kept.sum() == s.sum()


def test_capi_exports_every_declared_symbol():
    """liblbm.so loads without a GPU and exports each function of include/lbm.h."""
    import ctypes
    from flow_anizotropy_b200 import _lib
    hdr = (ROOT / "include" / "lbm.h").read_text()
    names = re.findall(r"^\s*(?:int|void|const char|long long)\s*\*?\s*(lbm_\w+)\s*\(", hdr, re.M)
    assert len(names) >= 18
    L = ctypes.CDLL(str(_lib.LIB_PATH))
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(_lib.SYMBOLS)
    assert L.lbm_version() == 1


def test_poisson_arrivals():
    from flow_anizotropy_b200.serve import poisson_arrivals
    a = poisson_arrivals(20.0, 100.0, seed=1)
    assert a == poisson_arrivals(20.0, 100.0, seed=1)
    assert all(x < y for x, y in zip(a, a[1:])) and a[-1] < 100.0
    assert 1800 < len(a) < 2200


class _FakeBatch:
    """Stand-in for solver.Batch: a request finishes after `cost` run() calls."""

    def __init__(self, cost=2, budget_slots=1000):
        self.cost, self.slots = cost, budget_slots
        self.left = {}
        self.order = []

    def submit(self, solid, forces, params, tag):
        if len(self.left) >= self.slots:
            return False
        self.left[tag] = self.cost
        self.order.append(tag)
        return True

    def run(self, chunks=1):
        for t in self.left:
            self.left[t] -= chunks

    def poll(self):
        done = [t for t, v in self.left.items() if v <= 0]
        for t in done:
            del self.left[t]
        return [(t, ["r"]) for t in done]

    def resident_bytes(self):
        return 0

    def close(self):
        pass


def test_server_admits_in_order_under_work_cap():
    """Continuous batching admits in arrival order, keeps the resident work
    (pore voxels x directions) under the cap, and always admits one request."""
    from flow_anizotropy_b200.serve import Server
    from flow_anizotropy_b200.solver import Params3D
    clock = iter(range(10**6)).__next__
    fake = _FakeBatch(cost=3)
    srv = Server(precision="fp32", batch=fake, max_work=3 * 100, clock=lambda: float(clock()))
    small = np.zeros((4, 5, 5), np.uint8)          # 100 pores
    big = np.zeros((8, 8, 8), np.uint8)            # 512 pores x 3 > cap: admitted alone
    forces = [[1e-6, 0, 0]]
    ids = [srv.submit(s, forces * 3 if s is big else forces, Params3D()) for s in (small, small, big, small)]
    seen_work = []
    while not srv.idle():
        srv.pump()
        seen_work.append(srv.resident_work)
        assert srv.resident_work <= 3 * 100 or len(srv.inflight) == 1
    assert fake.order == ids
    assert set(srv.results()) == set(ids)
    assert max(seen_work) > 0


def _dataset(tmp_path, shapes, seed=0):
    """A structures.csv dataset in the layout of the reference generator."""
    import pandas as pd
    from flow_anizotropy_b200 import structures as st
    from flow_anizotropy_b200.structure_io3d import save_structure
    d = tmp_path / "ds"
    (d / "structures").mkdir(parents=True)
    rows = []
    for i, shp in enumerate(shapes):
        solid = st.sphere_packing(shp, 3.0, 0.6, seed=seed + i, percolate=(True, True, True))
        name = f"s{i:04d}.raw"
        save_structure(d / "structures" / name, solid)
        rows.append({"sample_id": i, "filename": name, "group": "ab"[i % 2]})
    pd.DataFrame(rows).to_csv(d / "structures.csv", index=False)
    return d


def test_batch3d_plan_resume_and_atomic_rows(tmp_path):
    """Task planning (limit, shard, interleave), the resume rule (complete CSVs
    cached, incomplete ones removed and redone) and the atomic row write."""
    from flow_anizotropy_b200 import batch3d as B
    from flow_anizotropy_b200.solver import Result3D
    d = _dataset(tmp_path, [(10, 11, 12)] * 5)
    tasks = B.plan(str(d))
    assert [t.sample_id for t in tasks] == [0, 1, 2, 3, 4]
    assert tasks[0].structure == str(d / "structures" / "s0000.raw")
    assert tasks[0].out_csv == str(d / "perm" / "000000.csv")
    assert [t.sample_id for t in B.plan(str(d), shard="1/2")] == [1, 3]
    assert [t.sample_id for t in B.plan(str(d), limit=3)] == [0, 1, 2]
    assert [t.sample_id for t in B.plan(str(d), interleave="group")] == [0, 1, 2, 3, 4]
    cfg = B.solver_config("--eps 1e-6 --lag 500 --validate", "fp32")
    assert cfg["eps"] == 1e-6 and cfg["lag"] == 500 and cfg["validate"] and cfg["precision"] == "fp32"
    cfg["ff"] = 1.0
    (d / "perm").mkdir()
    solid = np.zeros((12, 11, 10), np.uint8)
    runs = [Result3D(q=np.array([1e-6 if c == j else 1e-9 for c in range(3)]), se=np.zeros(3), steps=5000,
                     converged=int(j != 2), status=0) for j in range(3)]
    assert B.write_row(tasks[0], cfg, solid, runs) == 3           # a direction did not converge
    assert B.valid_result(tasks[0].out_csv)
    assert not any(".tmp." in f for f in os.listdir(d / "perm"))
    Path(tasks[1].out_csv).write_text("filename,K_xx\n")         # left by a killed run
    work, cached = B.todo(tasks)
    assert [t.sample_id for t in cached] == [0]
    assert [t.sample_id for t in work] == [1, 2, 3, 4]
    assert not Path(tasks[1].out_csv).exists()


def test_block_criterion_sample_divides_lag():
    from flow_anizotropy_b200 import solver as S
    assert S.Params3D(lag=1000, precision="fp16").to_c().sample == 50
    assert S.Params3D(lag=120, precision="fp16").to_c().sample == 10      # gcd(120, 50)
    assert S.Params3D(lag=7, sample=3, precision="fp16").to_c().sample == 1
    for lag in (100, 120, 250, 333, 1000, 2000):
        s = S.Params3D(lag=lag).to_c().sample
        assert s > 0 and lag % s == 0


def test_criterion_codes():
    from flow_anizotropy_b200 import _lib
    from flow_anizotropy_b200 import solver as S
    assert S.Params3D(precision="fp16").to_c().criterion == _lib.CRIT_BATCH
    assert S.Params3D(precision="bf16").to_c().criterion == _lib.CRIT_BATCH
    assert S.Params3D(precision="fp32").to_c().criterion == _lib.CRIT_DRIFT
    assert S.Params3D(precision="fp64").to_c().criterion == _lib.CRIT_DRIFT
    assert S.Params3D(precision="fp16", criterion="block").to_c().criterion == _lib.CRIT_BLOCK
    assert S.Params3D(precision="fp32", criterion="batch").to_c().criterion == _lib.CRIT_BATCH
    assert S.Params3D().to_c().variant == _lib.LBM_VARIANT_DEFAULT
