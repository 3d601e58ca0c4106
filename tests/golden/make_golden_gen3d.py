"""Golden fixtures for the structure generator, from the REFERENCE generator.

    python tests/golden/make_golden_gen3d.py     (imports scripts/gen_aniso_structures3d.py
                                                  from the reference checkout)

Runs the reference's own per-sample generator (gen_one) for the first samples
of two seeds at a small cell size and commits what it wrote: the .raw
structures and their structures.csv rows (tests/golden/gen3d/).  The CPU
oracle (oracle/gen3d_oracle.py) and, on a GPU, flow_anizotropy_b200.gen3d are
checked against these.
"""
import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "gen3d"
REF_SCRIPTS = Path("/root/reference/scripts")

SIZE = 24
# (seed, sample ids, porosity range); the low-porosity case makes the
# reference redraw samples whose pore phase does not percolate
CASES = [(0, range(0, 6), (0.65, 0.90), 200), (7, range(0, 3), (0.65, 0.90), 200),
         (5, range(0, 4), (0.12, 0.18), 200), (5, range(0, 2), (0.08, 0.14), 5)]


def main():
    sys.path.insert(0, str(REF_SCRIPTS))
    import gen_aniso_structures3d as ref          # the reference generator
    OUT.mkdir(exist_ok=True)
    for f in OUT.glob("*.raw"):
        f.unlink()
    ref._init_worker(SIZE)
    rows = []
    for seed, ids, (plo, phi), attempts in CASES:
        cfg = {"structures_dir": str(OUT), "seed": seed, "k0_min": 3.0, "k0_max": 7.0, "dk": 1.0,
               "modes_min": 20, "modes_max": 80, "por_min": plo, "por_max": phi, "max_attempts": attempts}
        for i in ids:
            r = ref.gen_one(i, cfg)
            if r is None:                 # no percolating draw within max_attempts
                r = {"sample_id": i, "kept": False}
            else:
                r = {k: (v.item() if hasattr(v, "item") else v) for k, v in r.items()}
                r["kept"] = True
            r.update(seed=seed, por_min=plo, por_max=phi, max_attempts=attempts)
            rows.append(r)
    (OUT / "rows.json").write_text(json.dumps({"size": SIZE, "rows": rows}, indent=1) + "\n")
    print(f"wrote {len(rows)} structures to {OUT}")


if __name__ == "__main__":
    main()
