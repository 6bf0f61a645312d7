"""Golden fixtures for the skewed three-way join + group-by + top-k, computed
by the reference itself: run_q18 (compiled unchanged into ``oracle/_ref/``)
aggregates the joined rows.

The group-by's count per a_id is run_q18's dense sum_qty per orderkey
(bespoke_tpch/query_q18.cpp:205-262) when each joined B row becomes one
lineitem of quantity 1.00 with l_orderkey = its a_id
(``datagen.groupby_as_q18_tables``; the C filter and the join are plain numpy,
``datagen.groupby_joined_a_ids``).  QUANTITY "0" makes run_q18 return every
group, so its rows give the number of groups, the joined-row count (the sum of
the counts) and, ordered by (count desc, a_id asc), the top groups.  min(year)
has no counterpart in run_q18 and is not in these fixtures.

Each fixture records the ``datagen.gen_groupby`` call (sizes, seed), the query
and a SHA-256 of the generated columns, so a change of the generator is caught.

Run from the repository root where the reference harness is built:
    python tests/golden/make_golden_groupby.py
"""
from __future__ import annotations

import dataclasses
import hashlib
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from bespokeolap_artifacts_b200 import datagen as dg  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = Path(__file__).resolve().parent / "groupby_q18_reference.json"
TOP = 50

# (n_a, n_b, n_c, seed, variant); variant: None = the generator's own query,
# "cats<i>" = the i-th of three seeded category sets, "bad_ids" =
# datagen.groupby_with_bad_ids, "empty" = a year range nothing matches.
CASES = [
    (1000, 20_000, 5000, 1, None),
    (20_000, 300_000, 40_000, 2, None),
    (5000, 100_000, 20_000, 7, "bad_ids"),
    (1000, 50_000, 5000, 6, "empty"),
    (2_500_000, 36_000_000, 4_000_000, 3, None),
    (2_500_000, 36_000_000, 4_000_000, 3, "cats0"),
    (2_500_000, 36_000_000, 4_000_000, 3, "cats1"),
]


def query_sets(seed: int = 11) -> list[list[int]]:
    rng = np.random.default_rng(seed)
    return [sorted(int(v) for v in rng.choice(113, size=8, replace=False)) for _ in range(3)]


_BASE: dict = {}


def make_case(n_a: int, n_b: int, n_c: int, seed: int, variant):
    """The seeded input of one fixture (shared with the tests).  The last
    generated base input is kept, so the variants of one size share it."""
    key = (n_a, n_b, n_c, seed)
    if key not in _BASE:
        _BASE.clear()
        _BASE[key] = dg.gen_groupby(n_a, n_b, n_c, seed=seed)
    base = _BASE[key]
    g = dataclasses.replace(base, meta=dict(base.meta))
    if variant == "bad_ids":
        g = dataclasses.replace(g, b_a=base.b_a.copy(), b_c=base.b_c.copy())
        g = dg.groupby_with_bad_ids(g)
    elif variant == "empty":
        g.year_lo, g.year_hi = 3000, 3001
    elif variant and variant.startswith("cats"):
        g.cat_set = np.asarray(query_sets()[int(variant[4:])], dtype=np.uint16)
    return g


def input_sha(g) -> str:
    h = hashlib.sha256()
    for a in (g.a_ids, g.b_a, g.b_c, g.c_cat, g.c_year, np.asarray(g.cat_set, np.uint16),
              np.asarray([g.year_lo, g.year_hi], np.int64)):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def reference_groups(g) -> dict:
    tables = dg.groupby_as_q18_tables(g)
    db = O.RefDatabase(tables)
    try:
        keys, qty, _ = db.q18("0", tables["n_orders"])
    finally:
        db.close()
    assert np.all(qty % 100 == 0)
    counts = qty // 100
    order = np.lexsort((keys, -counts))
    return dict(n_groups=int(len(keys)), joined_rows=int(counts.sum()),
                keys=keys[order][:TOP].tolist(), counts=counts[order][:TOP].tolist())


def main():
    out = []
    for n_a, n_b, n_c, seed, variant in CASES:
        g = make_case(n_a, n_b, n_c, seed, variant)
        r = reference_groups(g)
        out.append(dict(gen="gen_groupby", n_a=n_a, n_b=n_b, n_c=n_c, seed=seed, variant=variant,
                        cat_set=[int(v) for v in g.cat_set], year_lo=g.year_lo, year_hi=g.year_hi,
                        input_sha256=input_sha(g), **r))
        print(n_a, n_b, n_c, seed, variant, r["n_groups"], r["joined_rows"], r["keys"][:3], flush=True)
    OUT.write_text(json.dumps(out, indent=1) + "\n")
    print("wrote", OUT.name)


if __name__ == "__main__":
    main()
