"""Pins the C restatement (oracle/bo_oracle.c) to the reference.

The reference ships no golden vectors, so the fixtures in tests/golden were
produced by the reference's own pipelines compiled unchanged
(tests/golden/make_golden.py).  These tests run on the CPU only.
"""
import json
from pathlib import Path

import numpy as np
import pytest

from bespokeolap_artifacts_b200 import datagen as dg
from oracle import oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden"
Q1_FIELDS = ("sum_qty", "sum_base_price", "sum_disc_price", "sum_charge", "avg_qty", "avg_price", "avg_disc")


def _q1_oracle_rows(t, delta):
    aggs, rc = O.q1_fact(t, dg.days_from_civil(1998, 12, 1) - delta)
    assert rc == 0
    rows = []
    for g, a in enumerate(aggs):
        if a["count"] == 0:
            continue
        rows.append((dg.FLAG_A_LETTERS[g // t.n_flag_b], dg.FLAG_B_LETTERS[g % t.n_flag_b], a))
    rows.sort(key=lambda r: (r[0], r[1]))
    return rows


@pytest.mark.parametrize("case", json.loads((GOLDEN / "q1_reference.json").read_text()),
                         ids=lambda c: f"seed{c['seed']}-n{c['n']}-d{c['delta']}")
def test_q1_oracle_matches_reference_golden(case):
    t = dg.gen_fact(case["n"], case["seed"])
    rows = _q1_oracle_rows(t, case["delta"])
    assert len(rows) == len(case["rows"])
    for (rf, ls, agg), ref in zip(rows, case["rows"]):
        assert (rf, ls) == (ref["returnflag"], ref["linestatus"])
        assert agg["count"] == ref["count_order"]
        got = O.q1_finalize(agg)
        for f, v in zip(Q1_FIELDS, got):
            assert v.hex() == ref[f], f  # bitwise-equal doubles


@pytest.mark.parametrize("case", json.loads((GOLDEN / "q3_reference.json").read_text()),
                         ids=lambda c: f"seed{c['seed']}")
def test_join_oracle_matches_reference_q3_golden(case):
    j = dg.gen_join(case["n_build"], case["n_probe"], case["seed"])
    r = O.join_agg(j)
    assert r["sum_trunc"] == case["revenue_sum"]
    assert r["match_count"] == case["lineitems_emitted"]


@pytest.mark.parametrize("case", json.loads((GOLDEN / "q6_reference.json").read_text()),
                         ids=lambda c: f"{c['date']}-{c['discount']}-{c['quantity']}")
def test_q6_oracle_matches_reference_golden(case):
    t = dg.gen_fact(case["n"], case["seed"])
    li = dg.fact_to_storage_plan(t)
    base = dg.days_from_civil(1992, 1, 1)
    y, m, d = map(int, case["date"].split("-"))
    start = dg.days_from_civil(y, m, d) - base
    end = dg.days_from_civil(y + 1, m, d) - base
    disc = round(float(case["discount"]) * 100)
    qty = round(float(case["quantity"]) * 100)
    rev, _ = O.q6_lineitem(li, start, end, disc - 1, disc + 1, qty)
    assert rev == case["revenue_raw"]



def test_q1_wide_and_storage_layout_oracles_agree():
    t = dg.gen_fact(50_000, 11)
    wide, rc = O.q1_fact(t, dg.Q1_CUTOFF)
    assert rc == 0
    narrow, rc = O.q1_lineitem(dg.fact_to_storage_plan(t), dg.Q1_CUTOFF - 8035, 6)
    assert rc == 0
    assert wide == narrow


def test_q1_oracle_against_numpy():
    t = dg.gen_fact(20_000, 12)
    aggs, _ = O.q1_fact(t, dg.Q1_CUTOFF)
    keep = t.ship_date <= dg.Q1_CUTOFF
    code = t.flag_a.astype(np.int64) * 2 + t.flag_b
    p1 = t.ext_price * (100 - t.discount)
    for g in range(6):
        m = keep & (code == g)
        a = aggs[g]
        assert a["count"] == int(m.sum())
        assert a["sum_qty"] == int(t.quantity[m].sum())
        assert a["sum_disc_price_exact"] == int(p1[m].sum())
        assert a["sum_disc_price"] == int((p1[m] // 100).sum())
        assert a["sum_charge_exact"] == sum(int(x) * (100 + int(y)) for x, y in zip(p1[m], t.tax[m]))


def test_join_oracle_against_numpy():
    j = dg.gen_join(5_000, 20_000, 13)
    r = O.join_agg(j)
    q = (j.b_date < j.date_lt) & (j.b_seg == j.seg_eq)
    keys = set(j.b_key[q].tolist())
    m = np.array([k in keys for k in j.p_fk.tolist()])
    p1 = j.p_price * (100 - j.p_disc)
    assert r["build_count"] == int(q.sum())
    assert r["match_count"] == int(m.sum())
    assert r["sum_exact"] == int(p1[m].sum())
    assert r["sum_trunc"] == int((p1[m] // 100).sum())


def test_groupby_oracle_against_pandas():
    pd = pytest.importorskip("pandas")
    g = dg.gen_groupby(20_000, 300_000, 40_000, seed=14)
    r = O.groupby_topk(g, k=25)
    cok = np.isin(g.c_cat, g.cat_set) & (g.c_year >= g.year_lo) & (g.c_year <= g.year_hi)
    sel = cok[g.b_c]
    df = pd.DataFrame({"a": g.b_a[sel], "y": g.c_year[g.b_c[sel]]})
    agg = df.groupby("a").agg(count=("y", "size"), min_year=("y", "min")).reset_index()
    agg = agg.sort_values(["count", "a"], ascending=[False, True]).head(25)
    assert r["n_groups"] == int(df["a"].nunique())
    assert r["joined_rows"] == int(sel.sum())
    assert r["keys"] == agg["a"].tolist()
    assert r["counts"] == agg["count"].tolist()
    assert r["min_years"] == agg["min_year"].tolist()


def test_radix_sort_oracle():
    rng = np.random.default_rng(15)
    k = rng.integers(0, 2**64, size=10_000, dtype=np.uint64)
    k[::7] = k[3]  # ties
    v = np.arange(10_000, dtype=np.uint32)
    sk, sv = O.radix_sort_pairs(k, v)
    order = np.argsort(k, kind="stable")
    assert np.array_equal(sk, k[order]) and np.array_equal(sv, v[order])


@pytest.mark.skipif(not O.ref_available(), reason="compiled reference harness not built")
@pytest.mark.parametrize("seed", [21, 22])
def test_q1_oracle_matches_live_reference(seed):
    t = dg.gen_fact(30_011, seed)
    db = O.RefDatabase(dg.fact_as_lineitem(t))
    ref, _ = db.q1(90)
    rows = _q1_oracle_rows(t, 90)
    for (rf, ls, agg), r in zip(rows, ref):
        assert (rf, ls, agg["count"]) == (r["returnflag"], r["linestatus"], r["count_order"])
        assert O.q1_finalize(agg) == [r[f] for f in Q1_FIELDS]
    # the builder's storage-plan columns fed to the storage-layout restatement
    li = db.lineitem()
    ng = li["returnflag_count"] * li["linestatus_count"]
    aggs, rc = O.q1_lineitem(li, dg.Q1_CUTOFF - li["base_date_days"], ng)
    assert rc == 0
    assert sum(a["count"] for a in aggs) == sum(r["count_order"] for r in ref)


@pytest.mark.skipif(not O.ref_available(trace=True), reason="compiled reference harness not built")
def test_join_oracle_matches_live_reference_q3():
    j = dg.gen_join(40_000, 160_000, 23)
    tables, args = dg.join_as_q3_tables(j)
    db = O.RefDatabase(tables, trace=True)
    r = db.q3(args["segment"], args["date"])
    o = O.join_agg(j)
    assert r["revenue_sum"] == o["sum_trunc"]
    assert r["trace"]["q3_lineitem_scan_rows_emitted"] == o["match_count"]


GB_CASES = json.loads((GOLDEN / "groupby_q18_reference.json").read_text())


def groupby_golden_input(case):
    """Regenerates a group-by fixture's input (tests/golden/make_golden_groupby.py)
    and checks it against the fixture's SHA-256."""
    import sys

    if str(GOLDEN) not in sys.path:
        sys.path.insert(0, str(GOLDEN))
    import make_golden_groupby as MG

    g = MG.make_case(case["n_a"], case["n_b"], case["n_c"], case["seed"], case["variant"])
    assert MG.input_sha(g) == case["input_sha256"], "the seeded generator changed: regenerate the fixtures"
    return g


@pytest.mark.parametrize("case", GB_CASES, ids=lambda c: f"b{c['n_b']}-seed{c['seed']}-{c['variant']}")
def test_groupby_oracle_matches_reference_q18_golden(case):
    """Counts, group count, joined rows and (count desc, a_id asc) order of the
    C restatement equal run_q18's dense aggregation of the same joined rows."""
    g = groupby_golden_input(case)
    r = O.groupby_topk(g, k=len(case["keys"]) or 1)
    assert r["n_groups"] == case["n_groups"]
    assert r["joined_rows"] == case["joined_rows"]
    assert r["keys"] == case["keys"]
    assert r["counts"] == case["counts"]
