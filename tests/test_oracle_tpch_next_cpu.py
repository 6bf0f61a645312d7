"""The numpy restatements behind the GPU tests of Q4, Q12 and Q14, pinned
against the reference itself: its own load / build / query (compiled
unchanged into oracle/_ref/ref_tpch_driver) answers the same requests on the
same seeded Parquet files, on the CPU.  Q12 runs on data with receipts up to
60 days after shipping, where the reference's shard pruning
(bespoke_tpch/query_q12.cpp:265-270, shards of builder_impl.cpp:855-911)
drops lineitems the plain filter would keep.  CPU only."""
import csv
import subprocess
from pathlib import Path

import numpy as np
import pyarrow.parquet as pq
import pytest

from tpch_parquet import write_tpch

ROOT = Path(__file__).resolve().parent.parent
REF_DRIVER = ROOT / "oracle" / "_ref" / "ref_tpch_driver"
D1992 = 8035  # 1992-01-01 in days since 1970-01-01


def days(col) -> np.ndarray:
    return col.to_numpy().astype("datetime64[D]").astype(np.int64) - D1992


def offset(date: str, months: int = 0) -> int:
    y, m, d = map(int, date.split("-"))
    m0 = m - 1 + months
    y, m = y + m0 // 12, m0 % 12 + 1
    dim = [31, 29 if (y % 4 == 0 and (y % 100 != 0 or y % 400 == 0)) else 28, 31, 30, 31, 30, 31, 31, 30, 31, 30,
           31][m - 1]
    return int((np.datetime64(f"{y:04d}-{m:02d}-{min(d, dim):02d}") - np.datetime64("1992-01-01")).astype(int))


def reference(data: Path, workdir: Path, requests: list[str]) -> list[list[list[str]]]:
    workdir.mkdir(parents=True, exist_ok=True)
    p = subprocess.run([str(REF_DRIVER), str(data) + "/"], input="\n".join(requests) + "\n\n", text=True,
                       capture_output=True, cwd=workdir, timeout=300)
    assert p.returncode == 0, p.stderr
    return [list(csv.reader(open(workdir / f"result{i + 1}.csv"))) for i in range(len(requests))]


@pytest.fixture(scope="module")
def tables(tmp_path_factory):
    if not REF_DRIVER.exists():
        pytest.skip("reference driver not built")
    d = write_tpch(tmp_path_factory.mktemp("tpch") / "d", n_customer=3000, n_orders=40000, seed=9, late_receipts=True)
    t = {n: pq.read_table(d / f"{n}.parquet") for n in ("lineitem", "orders", "part", "supplier")}
    return d, t


def scaled(col) -> np.ndarray:
    return np.round(col.to_numpy().astype(np.float64) * 100).astype(np.int64)


def q12(t, m1, m2, date, prune=True):
    L, O, S = t["lineitem"], t["orders"], t["supplier"]
    start, end = offset(date), offset(date, 12)
    ship, commit, receipt = days(L["l_shipdate"]), days(L["l_commitdate"]), days(L["l_receiptdate"])
    mode = np.array(L["l_shipmode"].to_pylist())
    ok = np.isin(mode, [m1, m2]) & (commit < receipt) & (ship < commit) & (receipt >= start) & (receipt < end)
    # shard pruning: shards of (ship year-month, discount, quantity / 100, supplier nation)
    ship_dt = (ship + D1992).astype("datetime64[D]")
    month_index = ship_dt.astype("datetime64[M]").astype(np.int64) + 1970 * 12
    nation = dict(zip(S["s_suppkey"].to_pylist(), S["s_nationkey"].to_pylist()))
    supp = np.array([nation.get(k, -1) for k in L["l_suppkey"].to_pylist()])
    key = (month_index << 24) | (scaled(L["l_discount"]) << 16) | ((scaled(L["l_quantity"]) // 100) << 8) | \
        np.where(supp >= 0, supp, 255)
    order = np.argsort(key, kind="stable")
    ks, ss = key[order], ship[order]
    starts = np.r_[0, np.flatnonzero(np.diff(ks)) + 1]
    shard_max = np.empty_like(ship)
    shard_max[order] = np.repeat(np.maximum.reduceat(ss, starts), np.diff(np.r_[starts, len(ks)]))
    if prune:
        ok &= shard_max >= start - 30
    prio = dict(zip(O["o_orderkey"].to_pylist(), O["o_orderpriority"].to_pylist()))
    rows = []
    for m in sorted({m1, m2}):
        sel = ok & (mode == m)
        p = [prio.get(k) for k in L["l_orderkey"].to_numpy()[sel]]
        p = [x for x in p if x is not None]
        high = sum(x in ("1-URGENT", "2-HIGH") for x in p)
        if p:
            rows.append([m, str(high), str(len(p) - high)])
    return rows


def q4(t, date):
    L, O = t["lineitem"], t["orders"]
    start, end = offset(date), offset(date, 3)
    late = days(L["l_commitdate"]) < days(L["l_receiptdate"])
    late_keys = set(L["l_orderkey"].to_numpy()[late].tolist())
    od = days(O["o_orderdate"])
    sel = (od >= start) & (od < end) & np.isin(O["o_orderkey"].to_numpy(), list(late_keys))
    pr = np.array(O["o_orderpriority"].to_pylist())[sel]
    vals, counts = np.unique(pr, return_counts=True)
    return [[v, str(c)] for v, c in zip(vals, counts)]


def q14(t, date):
    L, P = t["lineitem"], t["part"]
    start, end = offset(date), offset(date, 1)
    promo = {}
    for k, ty in zip(P["p_partkey"].to_pylist(), P["p_type"].to_pylist()):
        promo[k] = ty.startswith("PROMO")  # a later row of a key wins
    ship = days(L["l_shipdate"])
    price = scaled(L["l_extendedprice"])
    dprice = price * (100 - scaled(L["l_discount"])) // 100
    total = pr = 0
    for s, k, v in zip(ship, L["l_partkey"].to_pylist(), dprice):
        if start <= s < end and k in promo:
            total += int(v)
            pr += int(v) if promo[k] else 0
    return [[f"{100.0 * pr / total:.2f}" if total > 0 else "0.00"]]


def test_q12_q4_q14_restatements_match_the_reference(tables, tmp_path):
    data, t = tables
    reqs = ['12 "MODE_A" "MODE_C" "1994-01-01"', '12 "MODE_B" "MODE_F" "1996-03-31"', '4 "1993-07-01"',
            '4 "1996-11-30"', '14 "1995-09-01"', '14 "1993-02-28"']
    got = reference(data, tmp_path / "ref", reqs)
    assert got[0][1:] == [[f'{r[0]}', r[1], r[2]] for r in q12(t, "MODE_A", "MODE_C", "1994-01-01")]
    assert got[1][1:] == [[f'{r[0]}', r[1], r[2]] for r in q12(t, "MODE_B", "MODE_F", "1996-03-31")]
    assert got[2][1:] == q4(t, "1993-07-01")
    assert got[3][1:] == q4(t, "1996-11-30")
    assert got[4][1:] == q14(t, "1995-09-01")
    assert got[5][1:] == q14(t, "1993-02-28")
    # the pruning matters on this data: without it the first request's counts differ
    assert got[0][1:] != [[r[0], r[1], r[2]] for r in q12(t, "MODE_A", "MODE_C", "1994-01-01", prune=False)]
