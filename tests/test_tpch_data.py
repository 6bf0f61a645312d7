"""The seeded TPC-H-shaped Parquet writer: every table the reference's loader
reads (bespoke_tpch/loader_impl.cpp:12-19), and the options that select the
reference's code paths (late receipts for Q12's shard pruning, customer
nations inside the nation table for Q5, parts covering lineitem partkeys for
Q17).  CPU only."""
import numpy as np
import pyarrow.parquet as pq

from tpch_parquet import BRANDS, CONTAINERS, PRIORITIES, SHIPMODES, write_tpch  # noqa: F401

TABLES = ("customer", "lineitem", "nation", "orders", "part", "partsupp", "region", "supplier")


def days(col) -> np.ndarray:
    return col.to_numpy().astype("datetime64[D]").astype(np.int64)


def test_all_tables_and_defaults(tmp_path):
    d = write_tpch(tmp_path / "d", n_customer=300, n_orders=2000, seed=1)
    for t in TABLES:
        assert (d / f"{t}.parquet").exists()
    li = pq.read_table(d / "lineitem.parquet")
    lag = days(li["l_receiptdate"]) - days(li["l_shipdate"])
    assert lag.min() >= 1 and lag.max() <= 30
    assert set(li["l_shipmode"].to_pylist()) <= set(SHIPMODES)
    o = pq.read_table(d / "orders.parquet")
    assert set(o["o_orderpriority"].to_pylist()) <= set(PRIORITIES)
    c = pq.read_table(d / "customer.parquet")
    assert c["c_nationkey"].to_numpy().max() > 24  # nations without a nation row (Q10's unknown nations)
    p = pq.read_table(d / "part.parquet")["p_partkey"].to_numpy()
    assert len(p) == 151 and p[-1] == 3 and p[:-1].tolist() == list(range(1, 151))
    r = pq.read_table(d / "region.parquet")
    assert r["r_name"].to_pylist().count("REGION1") == 2


def test_options(tmp_path):
    d = write_tpch(tmp_path / "d", n_customer=300, n_orders=2000, seed=2, late_receipts=True,
                   customer_nations="known", n_supplier=25, n_part=199)
    li = pq.read_table(d / "lineitem.parquet")
    lag = days(li["l_receiptdate"]) - days(li["l_shipdate"])
    assert lag.max() > 30
    assert pq.read_table(d / "customer.parquet")["c_nationkey"].to_numpy().max() <= 24
    s = pq.read_table(d / "supplier.parquet")
    assert s["s_suppkey"].to_pylist() == list(range(1, 26))
    p = pq.read_table(d / "part.parquet")
    assert p["p_partkey"].to_numpy().max() >= li["l_partkey"].to_numpy().max()
    assert set(p["p_brand"].to_pylist()) <= set(BRANDS) and set(p["p_container"].to_pylist()) <= set(CONTAINERS)


def test_options_leave_the_other_columns_unchanged(tmp_path):
    a = write_tpch(tmp_path / "a", n_customer=300, n_orders=2000, seed=3)
    b = write_tpch(tmp_path / "b", n_customer=300, n_orders=2000, seed=3, late_receipts=True, n_supplier=25,
                   n_part=199)
    for t, cols in (("lineitem", ["l_orderkey", "l_quantity", "l_extendedprice", "l_shipdate", "l_returnflag"]),
                    ("orders", ["o_orderkey", "o_custkey", "o_orderdate", "o_comment"])):
        ta, tb = pq.read_table(a / f"{t}.parquet"), pq.read_table(b / f"{t}.parquet")
        for col in cols:
            assert ta[col].equals(tb[col]), (t, col)


def test_partsupp_lineitem_keys_and_part_layouts(tmp_path):
    """lineitem_keys="partsupp": every lineitem names one of its part's four
    partsupp pairs; repeat_part=False: n_part part rows and four partsupp rows
    per part (the layout run_q16 walks by row position); supplier comments
    with and without "Customer" before "Complaints", balances that vary."""
    d = write_tpch(tmp_path / "d", n_customer=300, n_orders=2000, seed=4, n_supplier=40, n_part=120,
                   repeat_part=False, lineitem_keys="partsupp")
    li, ps = pq.read_table(d / "lineitem.parquet"), pq.read_table(d / "partsupp.parquet")
    pairs = set(zip(ps["ps_partkey"].to_pylist(), ps["ps_suppkey"].to_pylist()))
    assert len(pairs) == ps.num_rows == 4 * 120
    assert all((p, s) in pairs for p, s in zip(li["l_partkey"].to_pylist(), li["l_suppkey"].to_pylist()))
    assert li["l_partkey"].to_numpy().max() <= 120 and len(set(li["l_partkey"].to_pylist())) > 100
    p = pq.read_table(d / "part.parquet")["p_partkey"].to_pylist()
    assert p == list(range(1, 121))
    s = pq.read_table(d / "supplier.parquet")
    comments = s["s_comment"].to_pylist()

    def banned(c):
        i = c.find("Customer")
        return i >= 0 and c.find("Complaints", i + 8) >= 0

    assert 0 < sum(map(banned, comments)) < len(comments)
    assert len(set(s["s_acctbal"].to_pylist())) > 30
    # the other columns do not move with these options
    base = write_tpch(tmp_path / "b", n_customer=300, n_orders=2000, seed=4, n_supplier=40, n_part=120)
    lb = pq.read_table(base / "lineitem.parquet")
    for col in ("l_orderkey", "l_quantity", "l_extendedprice", "l_discount", "l_shipdate"):
        assert li[col].equals(lb[col]), col
