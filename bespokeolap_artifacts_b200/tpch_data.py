"""Seeded TPC-H-shaped Parquet files (synthetic data) for the drop-in tests
and the bench's TPC-H section.

Writes the eight tables the reference's loader reads
(bespoke_tpch/loader_impl.cpp:12-19) with every column its builder reads, at
a small scale: customers with five market segments, nations, names,
addresses, phones and comments (some with quotes and commas), orders with
dates over 1992..1998, 1..7 lineitems per order sorted by orderkey with
TPC-H-like quantities, prices, discounts, taxes, flags and ship dates.
Decimal columns are DOUBLE, or DECIMAL(15,2) with decimal=True.

Key layouts (they select the reference's code paths):
  order_keys    "sparse": 8 of every 32 keys (the dbgen pattern);
                "dense": 1..n with key 1 dated first and key n last, so the
                date-sorted orders start at 1 and end at n while the rows in
                between are not in key order.
  customer_keys "dense": 1..n in order; "inner": 1, a shuffle of 2..n-1, n
                (first and last as dense, the rest not); "sparse": odd keys,
                shuffled, the last rows repeating earlier keys, and orders
                that name keys without a customer.
  shuffle_lineitem  lineitems in random order instead of by orderkey.
  late_receipts     receipt dates up to 60 days after shipping (TPC-H's are
                    at most 30), which the reference's Q12 shard pruning
                    notices.
  customer_nations  "wide": nationkeys 0..26, some without a nation row (Q10
                    drops those customers); "known": 0..24, inside the nation
                    table's key range (the reference's Q5 indexes its
                    per-nation arrays by the customer's nationkey unchecked).
  n_supplier        suppliers 1..n with nations 0..24 (default: one
                    supplier, key 1, nation 0).
  orderless_customers  custkeys divisible by 3 (but the largest order
                    custkey) place no order (Q22 counts customers without
                    orders); order custkeys keep the customers' key range,
                    which the reference's Q13 and Q22 index unchecked.
  n_part            parts 1..n (default 150; lineitems name parts 1..199).
                    The reference's Q17 reads its part bitmap at each
                    lineitem's partkey unchecked (query_q17.cpp:205-259), so
                    its parity data covers every lineitem partkey.
  lineitem_keys     "narrow": lineitems name parts 1..199 and suppliers 1..9;
                    "partsupp": each lineitem names one of the four
                    (partkey, suppkey) pairs of a random part 1..n_part, as in
                    TPC-H (a stream of its own).
  repeat_part       a last part row repeating key 3 with another type (the
                    later row wins); without it the part table has n_part
                    rows and partsupp four per part, the case the
                    reference's Q16 walks by row position
                    (query_q16.cpp:391-414).
Regions REGION0..REGION4 (keys 0..4; nations' regionkey = nationkey % 5) and
a later row repeating REGION1 with key 9.
Part names are three words of COLORS.  Ship modes MODE_A..MODE_G, AIR and AIR REG, ship
instructions from SHIPINSTRUCTS (one with trailing spaces), order statuses O, F and P, containers CONT_A..CONT_D and
Q19's twelve (a stream of their own for the instructions); order priorities 1-URGENT and 2-HIGH (the two the
reference's Q12 counts as high) and three others; part types with and
without the PROMO prefix Q14 looks for.  Commit dates 30..90 days
after the order, receipts 1..30 days after shipping.  These columns come from
a second seeded stream, so the other columns do not depend on them.
The nation table has keys 0..24 except 7; customers' nationkeys run 0..26.
Supplier comments are one to four words of SUPPLIER_WORDS (some contain
"Customer" before "Complaints", which Q16 bans, some the two the other way
round), supplier balances vary and manufacturers are MFGRS; these come from
streams of their own too.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pyarrow as pa
import pyarrow.parquet as pq

SEGMENTS = ["SEG_A", "SEG_B", "SEG_C", "SEG_D", "SEG_E"]
WORDS = ["ironic", "quick", "pending", "bold", 'say "hi"', "a,b", "deposits", "", "x\"y", "final"]
# the two ship modes, the ship instruction and the container lists run_q19
# compares against (bespoke_tpch/query_q19.cpp:160-179, 203-208), among others
SHIPMODES = ["MODE_A", "MODE_B", "MODE_C", "MODE_D", "MODE_E", "MODE_F", "MODE_G", "AIR", "AIR REG"]
STATUSES = ["O", "F", "P"]  # run_q21 walks the orders of status "F" (query_q21.cpp:166-178)
SHIPINSTRUCTS = ["DELIVER IN PERSON", "LEAVE AT DOOR", "HOLD AT DEPOT", "DELIVER IN PERSON  "]
Q19_CONTAINERS = ["SM CASE", "SM BOX", "SM PACK", "SM PKG", "MED BAG", "MED BOX", "MED PKG", "MED PACK",
                  "LG CASE", "LG BOX", "LG PACK", "LG PKG"]
PRIORITIES = ["1-URGENT", "2-HIGH", "3-PRIO_C", "4-PRIO_D", "5-PRIO_E"]
PART_TYPES = ["PROMO_A", "PROMO_B", "STD_A", "STD_B", "ECO_A", "PROMOTION", "PROM", "LARGE_PROMO"]
BRANDS = ["BRAND_A", "BRAND_B", "BRAND_C", "BRAND_D", "BRAND_E"]
# part-name words (Q9 looks for a substring of the name)
COLORS = ["amber", "azure", "cobalt", "coral", "crimson", "ivory", "jade", "khaki", "lilac", "maroon", "ochre",
          "olive", "pearl", "plum", "rust", "sage", "sand", "slate", "teal", "umber"]
CONTAINERS = ["CONT_A", "CONT_B", "CONT_C", "CONT_D"] + Q19_CONTAINERS
# supplier-comment words: run_q16 bans suppliers whose comment has "Customer"
# and, after it, "Complaints" (bespoke_tpch/query_q16.cpp:58-67)
SUPPLIER_WORDS = ["ironic", "Customer", "Complaints", "Customer Complaints", "requests", "Complaints Customer",
                  "CustomerComplaints", "carefully", "Customer Complaint", "say \"hi\""]
MFGRS = ["Manufacturer#1", "Manufacturer#2", "Manufacturer#3", "Manufacturer#4", "Manufacturer#5"]
D1992 = 8035  # 1992-01-01 in days since 1970-01-01


def _dec(values: np.ndarray, decimal: bool) -> pa.Array:
    if not decimal:
        return pa.array(values, pa.float64())
    from decimal import Decimal

    return pa.array([Decimal(f"{v:.2f}") for v in values], pa.decimal128(15, 2))


def _nations(keys: np.ndarray, mode: str) -> np.ndarray:
    """Customer nationkeys: "wide" 0..26 (25 and 26 have no nation row), or
    "known" within the nation table's key range 0..24."""
    if mode == "wide":
        return keys.astype(np.int32)
    if mode == "known":
        return (keys % 25).astype(np.int32)
    raise ValueError(mode)


def _text(rng, n: int, words: int) -> list[str]:
    picks = rng.integers(0, len(WORDS), (n, words))
    return [" ".join(WORDS[i] for i in row) for row in picks]


def _ragged_text(rng, n: int, max_words: int) -> list[str]:
    counts = rng.integers(0, max_words + 1, n)
    return [" ".join(WORDS[i] for i in rng.integers(0, len(WORDS), c)) for c in counts]


def write_tpch(out: Path, n_customer: int = 1500, n_orders: int = 15000, seed: int = 0,
               decimal: bool = False, order_keys: str = "sparse", customer_keys: str = "dense",
               shuffle_lineitem: bool = False, late_receipts: bool = False, customer_nations: str = "wide",
               n_supplier: int = 1, n_part: int = 150, orderless_customers: bool = False,
               repeat_part: bool = True, lineitem_keys: str = "narrow") -> Path:
    rng = np.random.default_rng(seed)
    rng2 = np.random.default_rng([seed, 12])
    out.mkdir(parents=True, exist_ok=True)
    if customer_keys == "dense":
        custkey = np.arange(1, n_customer + 1, dtype=np.int32)
    elif customer_keys == "inner":
        custkey = np.concatenate([[1], rng.permutation(np.arange(2, n_customer)), [n_customer]]).astype(np.int32)
    elif customer_keys == "sparse":
        custkey = rng.permutation(np.arange(n_customer, dtype=np.int32) * 2 + 1)
        custkey[-5:] = custkey[:5]  # repeated keys: the last row of each wins
    else:
        raise ValueError(customer_keys)
    seg = rng.integers(0, 5, n_customer)
    pq.write_table(pa.table({
        "c_custkey": custkey, "c_name": [f"Customer#{k:09d}" for k in custkey],
        "c_address": _text(rng, n_customer, 2), "c_nationkey": _nations(rng.integers(0, 27, n_customer), customer_nations),
        "c_phone": [f"{10 + a}-{b:03d}-{c:03d}-{d:04d}" for a, b, c, d in
                    zip(*(rng.integers(0, m, n_customer) for m in (25, 1000, 1000, 10000)))],
        "c_acctbal": _dec(rng.integers(-99999, 999999, n_customer) / 100.0, decimal),
        "c_mktsegment": [SEGMENTS[s] for s in seg], "c_comment": _text(rng, n_customer, 3),
    }), out / "customer.parquet")
    # dates 1992-01-01 .. 1998-08-02
    o_date = rng.integers(D1992, D1992 + 2405, n_orders).astype(np.int32)
    if order_keys == "sparse":  # TPC-H orderkeys: 8 of every 32
        orderkey = (np.arange(n_orders, dtype=np.int64) // 8 * 32 + np.arange(n_orders) % 8 + 1).astype(np.int32)
    elif order_keys == "dense":
        orderkey = np.arange(1, n_orders + 1, dtype=np.int32)
        o_date[0], o_date[-1] = D1992, D1992 + 2404
    else:
        raise ValueError(order_keys)
    if customer_keys == "sparse":
        o_cust = rng.choice(np.concatenate([custkey, custkey[:50] - 1]), n_orders).astype(np.int32)
    else:
        o_cust = rng.integers(1, n_customer + 1, n_orders).astype(np.int32)
    if orderless_customers:
        # custkeys divisible by 3 (but the largest) place no order: their orders
        # go to the key below, so order custkeys keep the customers' key range
        top = o_cust.max()
        o_cust = np.where((o_cust % 3 == 0) & (o_cust != top), o_cust - 1, o_cust).astype(np.int32)
    pq.write_table(pa.table({
        "o_orderkey": orderkey, "o_custkey": o_cust,
        "o_orderstatus": [STATUSES[i] for i in np.random.default_rng([seed, 17]).integers(0, 3, n_orders)],
        "o_totalprice": _dec(rng.integers(100000, 50000000, n_orders) / 100.0, decimal),
        "o_orderdate": pa.array(o_date, pa.date32()),
        "o_orderpriority": [PRIORITIES[i] for i in rng2.integers(0, len(PRIORITIES), n_orders)],
        "o_clerk": ["Clerk#000000001"] * n_orders, "o_shippriority": np.zeros(n_orders, np.int32),
        "o_comment": _ragged_text(rng, n_orders, 8),
    }), out / "orders.parquet")
    lines = rng.integers(1, 8, n_orders)
    lk = np.repeat(orderkey, lines)
    ld = np.repeat(o_date, lines)
    n = len(lk)
    qty = rng.integers(1, 51, n)
    price = qty * rng.integers(90000, 210000, n) / 100.0
    ship = ld + rng.integers(1, 122, n)
    rf = np.where(ship <= D1992 + 1267, np.array(["R", "A"])[rng.integers(0, 2, n)], "N")  # before / after 1995-06-17
    ls = np.where(ship > D1992 + 1267, "O", "F")
    commit = ld + rng2.integers(30, 91, n)
    receipt = ship + rng2.integers(1, 61 if late_receipts else 31, n)
    mode = rng2.integers(0, len(SHIPMODES), n)
    if shuffle_lineitem:
        perm = rng.permutation(n)
        lk, ld, qty, price, ship, rf, ls, commit, receipt, mode = (
            a[perm] for a in (lk, ld, qty, price, ship, rf, ls, commit, receipt, mode))
    l_part = rng.integers(1, 200, n).astype(np.int32)
    l_supp = rng.integers(1, 10, n).astype(np.int32)
    ns_ = max(n_supplier, 1)
    if lineitem_keys == "partsupp":  # a partsupp pair of a random part (the four below)
        rng7 = np.random.default_rng([seed, 21])
        l_part = rng7.integers(1, n_part + 1, n).astype(np.int32)
        j = rng7.integers(0, 4, n)
        l_supp = ((l_part - 1 + j * (ns_ // 4 + 1)) % ns_ + 1).astype(np.int32)
    elif lineitem_keys != "narrow":
        raise ValueError(lineitem_keys)
    pq.write_table(pa.table({
        "l_orderkey": lk, "l_partkey": l_part,
        "l_suppkey": l_supp, "l_linenumber": np.ones(n, np.int32),
        "l_quantity": _dec(qty.astype(np.float64), decimal), "l_extendedprice": _dec(price, decimal),
        "l_discount": _dec(rng.integers(0, 11, n) / 100.0, decimal), "l_tax": _dec(rng.integers(0, 9, n) / 100.0, decimal),
        "l_returnflag": rf.tolist(), "l_linestatus": ls.tolist(),
        "l_shipdate": pa.array(ship.astype(np.int32), pa.date32()),
        "l_commitdate": pa.array(commit.astype(np.int32), pa.date32()),
        "l_receiptdate": pa.array(receipt.astype(np.int32), pa.date32()),
        "l_shipinstruct": [SHIPINSTRUCTS[i] for i in np.random.default_rng([seed, 16]).integers(0, 4, n)],
        "l_shipmode": [SHIPMODES[i] for i in mode],
        "l_comment": [""] * n,
    }), out / "lineitem.parquet")
    one = np.ones(1, np.int32)
    # parts 1..n_part (lineitems name 1..199, so by default some have no part)
    # and a last row repeating key 3 with another type (the later row wins)
    rng3 = np.random.default_rng([seed, 14])
    pkey = np.concatenate([np.arange(1, n_part + 1), [3] if repeat_part else []]).astype(np.int32)
    rows_p = len(pkey)
    ptype = [PART_TYPES[i] for i in rng3.integers(0, len(PART_TYPES), rows_p)]
    if repeat_part:
        ptype[-1] = "STD_A" if ptype[2].startswith("PROMO") else "PROMO_B"
    psize = rng3.integers(1, 51, rows_p).astype(np.int32)
    pbrand = [BRANDS[i] for i in rng3.integers(0, len(BRANDS), rows_p)]
    pcont = [CONTAINERS[i] for i in rng3.integers(0, len(CONTAINERS), rows_p)]
    # names of three words from COLORS (a stream of their own, so the other
    # part columns do not depend on them)
    rng5 = np.random.default_rng([seed, 15])
    pname = [" ".join(COLORS[i] for i in row) for row in rng5.integers(0, len(COLORS), (rows_p, 3))]
    pmfgr = [MFGRS[i] for i in np.random.default_rng([seed, 20]).integers(0, len(MFGRS), rows_p)]
    pq.write_table(pa.table({"p_partkey": pkey, "p_name": pname, "p_mfgr": pmfgr,
                             "p_brand": pbrand, "p_type": ptype, "p_size": psize, "p_container": pcont,
                             "p_retailprice": _dec(np.ones(rows_p), decimal), "p_comment": [""] * rows_p}),
                   out / "part.parquet")
    if n_supplier <= 1:
        skey, snation = one, one * 0
    else:
        skey = np.arange(1, n_supplier + 1, dtype=np.int32)
        snation = np.random.default_rng([seed, 5]).integers(0, 25, n_supplier).astype(np.int32)
    ns = len(skey)
    rng6 = np.random.default_rng([seed, 18])
    s_comment = [" ".join(SUPPLIER_WORDS[i] for i in rng6.integers(0, len(SUPPLIER_WORDS), c))
                 for c in rng6.integers(1, 5, ns)]
    s_acctbal = np.random.default_rng([seed, 19]).integers(-99999, 999999, ns) / 100.0
    pq.write_table(pa.table({"s_suppkey": skey, "s_name": [f"Supplier#{k:09d}" for k in skey],
                             "s_address": [f"addr {k}, \"{k % 7}\"" for k in skey], "s_nationkey": snation,
                             "s_phone": [f"{10 + k % 25}-{k:03d}-000-0000" for k in skey],
                             "s_acctbal": _dec(s_acctbal, decimal), "s_comment": s_comment}),
                   out / "supplier.parquet")
    # four suppliers per part (key 1..n_part), rows in random order
    rng4 = np.random.default_rng([seed, 11])
    ps_part = np.repeat(np.arange(1, n_part + 1), 4)
    ps_supp = ((ps_part - 1 + np.tile(np.arange(4), n_part) * (ns // 4 + 1)) % ns + 1)
    perm = rng4.permutation(len(ps_part))
    n_ps = len(ps_part)
    pq.write_table(pa.table({"ps_partkey": ps_part[perm].astype(np.int32), "ps_suppkey": skey[ps_supp[perm] - 1],
                             "ps_availqty": rng4.integers(1, 10_000, n_ps).astype(np.int32),
                             "ps_supplycost": _dec(rng4.integers(100, 100_001, n_ps) / 100.0, decimal),
                             "ps_comment": [""] * n_ps}), out / "partsupp.parquet")
    nkey = np.array([k for k in range(25) if k != 7], np.int32)
    pq.write_table(pa.table({"n_nationkey": nkey, "n_name": [f"NATION_{k:02d}" for k in nkey],
                             "n_regionkey": nkey % 5, "n_comment": [""] * len(nkey)}), out / "nation.parquet")
    # five regions and a later row repeating a name (the first row of a name wins)
    pq.write_table(pa.table({"r_regionkey": np.array([0, 1, 2, 3, 4, 9], np.int32),
                             "r_name": [f"REGION{k}" for k in range(5)] + ["REGION1"], "r_comment": [""] * 6}),
                   out / "region.parquet")
    return out
