"""Generates the golden fixtures in this directory by running the reference's
own pipelines (compiled unchanged into ``oracle/_ref/``) on small seeded inputs.

The inputs are not stored: each fixture records the ``datagen`` call (function,
sizes, seed) that regenerates them, and the reference's outputs.  Doubles are
stored with ``float.hex`` so bitwise comparisons survive JSON.

Run from the repository root where the reference harness is built:
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from bespokeolap_artifacts_b200 import datagen as dg  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = Path(__file__).resolve().parent

Q1_CASES = [(1, 100_000), (2, 4_099), (3, 1), (4, 7)]
Q1_DELTAS = [90, 60, 3000]
Q3_CASES = [(5, 20_000, 80_000), (6, 1_000, 4_003), (7, 3, 10)]
Q6_CASES = [(8, 50_000)]
Q6_PARAMS = [("1994-02-01", "0.07", "23"), ("1996-01-01", "0.02", "40"), ("1992-03-15", "0.09", "10")]


def q1_fixture():
    out = []
    for seed, n in Q1_CASES:
        t = dg.gen_fact(n, seed)
        db = O.RefDatabase(dg.fact_as_lineitem(t))
        for delta in Q1_DELTAS:
            rows, _ = db.q1(delta)
            out.append(dict(gen="gen_fact", n=n, seed=seed, delta=delta, rows=[
                {k: (v.hex() if isinstance(v, float) else v) for k, v in r.items()} for r in rows]))
        db.close()
    return out


def q3_fixture():
    out = []
    for seed, nb, npr in Q3_CASES:
        j = dg.gen_join(nb, npr, seed)
        tables, args = dg.join_as_q3_tables(j)
        db = O.RefDatabase(tables, trace=True)
        r = db.q3(args["segment"], args["date"])
        out.append(dict(gen="gen_join", n_build=nb, n_probe=npr, seed=seed, segment=args["segment"],
                        date=args["date"], n_rows=r["n_rows"], revenue_sum=r["revenue_sum"],
                        lineitems_emitted=r["trace"]["q3_lineitem_scan_rows_emitted"],
                        orders_emitted=r["trace"]["q3_orders_scan_rows_emitted"]))
        db.close()
    return out


def q6_fixture():
    out = []
    for seed, n in Q6_CASES:
        t = dg.gen_fact(n, seed)
        db = O.RefDatabase(dg.fact_as_lineitem(t))
        for date, disc, qty in Q6_PARAMS:
            rev, _ = db.q6(date, disc, qty)
            out.append(dict(gen="gen_fact", n=n, seed=seed, date=date, discount=disc, quantity=qty,
                            revenue_raw=rev))
        db.close()
    return out


if __name__ == "__main__":
    (OUT / "q1_reference.json").write_text(json.dumps(q1_fixture(), indent=1) + "\n")
    (OUT / "q3_reference.json").write_text(json.dumps(q3_fixture(), indent=1) + "\n")
    (OUT / "q6_reference.json").write_text(json.dumps(q6_fixture(), indent=1) + "\n")
    print("wrote", sorted(p.name for p in OUT.glob("*.json")))
