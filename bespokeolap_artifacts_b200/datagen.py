"""Seeded synthetic inputs with the shapes, sizes and value distributions of the
engine's three pipeline workloads.  Nothing here comes from a benchmark's data:
every column is drawn from ``numpy.random.default_rng(seed)``.

* :func:`gen_fact`     -- scan-filter-group-aggregate fact table (6,000,000 rows
  at full size; wide layout, 38 B/row);
* :func:`gen_join`     -- filtered join: 1,500,000-row build side, 6,000,000-row
  probe side;
* :func:`gen_groupby`  -- skewed three-way join: A 2,500,000 ids, B 36,000,000
  (a_id, c_id) pairs drawn from bounded Zipf laws, C 4,000,000 rows.

Dates are days since 1970-01-01.  Money columns are fixed-point x100.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

DATE_LO = 8035    # 1992-01-01
DATE_HI = 10591   # 1998-12-31


def days_from_civil(y: int, m: int, d: int) -> int:
    """Days since 1970-01-01 of a proleptic Gregorian date (the era/day-of-era
    algorithm the reference uses, bespoke_tpch/query_q1.cpp:19-26)."""
    y -= m <= 2
    era = (y if y >= 0 else y - 399) // 400
    yoe = y - era * 400
    doy = (153 * (m + (-3 if m > 2 else 9)) + 2) // 5 + d - 1
    doe = yoe * 365 + yoe // 4 - yoe // 100 + doy
    return era * 146097 + doe - 719468


def civil_from_days(z: int) -> tuple[int, int, int]:
    """Inverse of :func:`days_from_civil` (bespoke_tpch/query_q3.cpp:27-38)."""
    z += 719468
    era = (z if z >= 0 else z - 146096) // 146097
    doe = z - era * 146097
    yoe = (doe - doe // 1460 + doe // 36524 - doe // 146096) // 365
    y = yoe + era * 400
    doy = doe - (365 * yoe + yoe // 4 - yoe // 100)
    mp = (5 * doy + 2) // 153
    d = doy - (153 * mp + 2) // 5 + 1
    m = mp + (3 if mp < 10 else -9)
    return y + (m <= 2), m, d


def date_string(days: int) -> str:
    y, m, d = civil_from_days(days)
    return f"{y:04d}-{m:02d}-{d:02d}"


Q1_DELTA = 90
Q1_CUTOFF = days_from_civil(1998, 12, 1) - Q1_DELTA   # 10471


# ------------------------------------------------------------ scan / agg ----
@dataclass
class FactTable:
    ship_date: np.ndarray   # int32 days
    quantity: np.ndarray    # int64 x100
    ext_price: np.ndarray   # int64 x100
    discount: np.ndarray    # int64 x100 (0..10)
    tax: np.ndarray         # int64 x100 (0..8)
    flag_a: np.ndarray      # uint8 {0,1,2}
    flag_b: np.ndarray      # uint8 {0,1}
    n_flag_a: int = 3
    n_flag_b: int = 2
    seed: int = 0

    @property
    def n_rows(self) -> int:
        return int(self.ship_date.shape[0])

    def columns(self):
        return [self.ship_date, self.quantity, self.ext_price, self.discount, self.tax, self.flag_a, self.flag_b]

    BYTES_PER_ROW = 4 + 8 + 8 + 8 + 8 + 1 + 1


def gen_fact(n: int = 6_000_000, seed: int = 0) -> FactTable:
    rng = np.random.default_rng(seed)
    return FactTable(
        ship_date=rng.integers(DATE_LO, DATE_HI, size=n, endpoint=True, dtype=np.int32),
        quantity=rng.integers(1, 50, size=n, endpoint=True, dtype=np.int64) * 100,
        ext_price=rng.integers(90_000, 10_500_000, size=n, endpoint=True, dtype=np.int64),
        discount=rng.integers(0, 10, size=n, endpoint=True, dtype=np.int64),
        tax=rng.integers(0, 8, size=n, endpoint=True, dtype=np.int64),
        flag_a=rng.integers(0, 2, size=n, endpoint=True, dtype=np.uint8),
        flag_b=rng.integers(0, 1, size=n, endpoint=True, dtype=np.uint8),
        seed=seed,
    )


# ------------------------------------------------------------------ join ----
@dataclass
class JoinInput:
    b_key: np.ndarray      # int32 unique keys 1..n_build, shuffled
    b_date: np.ndarray     # int32 days
    b_seg: np.ndarray      # uint8 0..4
    p_fk: np.ndarray       # int32 uniform over build keys
    p_price: np.ndarray    # int64 x100
    p_disc: np.ndarray     # int64 x100 0..10
    date_lt: int           # build filter: date < date_lt
    seg_eq: int            # build filter: segment == seg_eq
    seed: int = 0

    @property
    def n_build(self) -> int:
        return int(self.b_key.shape[0])

    @property
    def n_probe(self) -> int:
        return int(self.p_fk.shape[0])

    BUILD_BYTES_PER_ROW = 4 + 4 + 1
    PROBE_BYTES_PER_ROW = 4 + 8 + 8

    def algorithmic_bytes(self) -> int:
        return self.n_build * self.BUILD_BYTES_PER_ROW + self.n_probe * self.PROBE_BYTES_PER_ROW


def join_date_cutoff(selectivity: float = 0.2) -> int:
    return DATE_LO + int(selectivity * (DATE_HI - DATE_LO))


def gen_join(n_build: int = 1_500_000, n_probe: int = 6_000_000, seed: int = 0,
             date_lt: int | None = None, seg_eq: int | None = None) -> JoinInput:
    rng = np.random.default_rng(seed)
    key = rng.permutation(np.arange(1, n_build + 1, dtype=np.int32))
    date = rng.integers(DATE_LO, DATE_HI, size=n_build, endpoint=True, dtype=np.int32)
    seg = rng.integers(0, 4, size=n_build, endpoint=True, dtype=np.uint8)
    fk = rng.integers(1, max(n_build, 1), size=n_probe, endpoint=True, dtype=np.int32)
    price = rng.integers(90_000, 10_500_000, size=n_probe, endpoint=True, dtype=np.int64)
    disc = rng.integers(0, 10, size=n_probe, endpoint=True, dtype=np.int64)
    s = int(rng.integers(0, 4, endpoint=True)) if seg_eq is None else seg_eq
    d = join_date_cutoff() if date_lt is None else date_lt
    return JoinInput(key, date, seg, fk, price, disc, d, s, seed)


# --------------------------------------------------------------- group-by ----
def zipf_ranks(rng: np.random.Generator, n: int, n_ranks: int, s: float, chunk: int = 4_000_000) -> np.ndarray:
    """n draws of a bounded Zipf law over ranks 0..n_ranks-1 (P(r) ~ (r+1)^-s),
    by inverse CDF: a uniform draw is located in the cumulative weights."""
    w = np.arange(1, n_ranks + 1, dtype=np.float64) ** (-s)
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    out = np.empty(n, dtype=np.int64)
    for lo in range(0, n, chunk):
        hi = min(n, lo + chunk)
        idx = np.searchsorted(cdf, rng.random(hi - lo), side="right")
        np.minimum(idx, n_ranks - 1, out=idx)
        out[lo:hi] = idx
    return out


@dataclass
class GroupByInput:
    a_ids: np.ndarray      # int32 ids of A (1..n_a, shuffled)
    b_a: np.ndarray        # int32 a_id per B row (Zipf s_a over A, ranks -> ids by a seeded permutation)
    b_c: np.ndarray        # int32 c_id per B row (Zipf s_c over C rows, ranks -> rows by a seeded permutation)
    c_cat: np.ndarray      # uint16 category 0..112 (C row index is the c_id)
    c_year: np.ndarray     # int32 year 1900..2020
    cat_set: np.ndarray    # uint16, 8 distinct categories
    year_lo: int
    year_hi: int
    k: int = 10
    seed: int = 0
    meta: dict = field(default_factory=dict)

    @property
    def n_rows(self) -> int:
        return int(self.a_ids.shape[0] + self.b_a.shape[0] + self.c_cat.shape[0])

    def algorithmic_bytes(self) -> int:
        return self.a_ids.nbytes + self.b_a.nbytes + self.b_c.nbytes + self.c_cat.nbytes + self.c_year.nbytes


def gen_groupby(n_a: int = 2_500_000, n_b: int = 36_000_000, n_c: int = 4_000_000, seed: int = 0,
                s_a: float = 1.1, s_c: float = 0.9, n_cat_values: int = 113, n_cat_set: int = 8,
                year_lo: int = 1990, year_hi: int = 2010, k: int = 10) -> GroupByInput:
    rng = np.random.default_rng(seed)
    a_ids = rng.permutation(np.arange(1, n_a + 1, dtype=np.int32))
    rank_to_a = rng.permutation(np.arange(1, n_a + 1, dtype=np.int32))
    rank_to_c = rng.permutation(np.arange(0, n_c, dtype=np.int32))
    b_a = rank_to_a[zipf_ranks(rng, n_b, n_a, s_a)]
    b_c = rank_to_c[zipf_ranks(rng, n_b, n_c, s_c)]
    c_cat = rng.integers(0, n_cat_values - 1, size=n_c, endpoint=True, dtype=np.uint16)
    c_year = rng.integers(1900, 2020, size=n_c, endpoint=True, dtype=np.int32)
    cat_set = np.sort(rng.choice(n_cat_values, size=n_cat_set, replace=False)).astype(np.uint16)
    return GroupByInput(a_ids, b_a, b_c, c_cat, c_year, cat_set, year_lo, year_hi, k, seed,
                        meta={"s_a": s_a, "s_c": s_c, "rank_to_id": "seeded permutation"})


def fact_to_storage_plan(t: FactTable, base_date_days: int = DATE_LO) -> dict:
    """The reference builder's storage-plan lineitem columns for a fact table
    (bespoke_tpch/builder_impl.cpp:522-565): int16 date offsets, int32 prices,
    the truncated discounted_price, uint8 discount / tax, int16 quantity and the
    group code flag_a * n_flag_b + flag_b (codes in flag order)."""
    return dict(
        shipdate=(t.ship_date - base_date_days).astype(np.int16),
        returnflag_linestatus=(t.flag_a.astype(np.int32) * t.n_flag_b + t.flag_b).astype(np.uint8),
        extendedprice=t.ext_price.astype(np.int32),
        discounted_price=(t.ext_price * (100 - t.discount) // 100).astype(np.int32),
        discount=t.discount.astype(np.uint8),
        tax=t.tax.astype(np.uint8),
        quantity=t.quantity.astype(np.int16),
        n_rows=t.n_rows,
        base_date_days=base_date_days,
        returnflag_dict=FLAG_A_LETTERS[:t.n_flag_a],
        linestatus_dict=FLAG_B_LETTERS[:t.n_flag_b],
    )


# ---------------------------------------------- reference-table mappings ----
FLAG_A_LETTERS = "ABCDEFGH"   # flag_a code -> returnflag string (order-preserving)
FLAG_B_LETTERS = "VWXYZ"      # flag_b code -> linestatus string (order-preserving)


def fact_as_lineitem(t: FactTable) -> dict:
    """Maps the fact table onto the reference lineitem columns run_q1 reads:
    decimals as their decimal values (the reference builder scales them by 100
    with llround), flags as returnflag / linestatus letters whose string order
    equals the code order."""
    n = t.n_rows
    return dict(
        n_lineitem=n,
        l_orderkey=np.ones(n, dtype=np.int32),
        l_shipdate=t.ship_date,
        l_quantity=t.quantity / 100.0,
        l_extendedprice=t.ext_price / 100.0,
        l_discount=t.discount / 100.0,
        l_tax=t.tax / 100.0,
        l_returnflag=t.flag_a,
        l_linestatus=t.flag_b,
        n_orders=1, o_orderkey=np.ones(1, np.int32), o_custkey=np.ones(1, np.int32),
        o_orderdate=np.full(1, DATE_LO, np.int32),
        n_customer=1, c_custkey=np.ones(1, np.int32), c_mktsegment=np.zeros(1, np.uint8),
    )


def join_as_q3_tables(j: JoinInput) -> tuple[dict, dict]:
    """Maps the filtered join onto run_q3's tables (bespoke_tpch/query_q3.cpp:153):
    one customer and one order per build row (custkey = orderkey = key,
    mktsegment = segment, orderdate = date), lineitems = probe rows sorted by
    foreign key with a ship date after every cutoff.  run_q3 then sums
    trunc(price*(100-disc)/100) over exactly the matching probe rows.  Returns
    (tables, query args)."""
    order = np.argsort(j.p_fk, kind="stable")
    n = j.n_probe
    tables = dict(
        n_lineitem=n,
        l_orderkey=np.ascontiguousarray(j.p_fk[order]),
        l_shipdate=np.full(n, DATE_HI, np.int32),
        l_quantity=np.ones(n, np.float64),
        l_extendedprice=j.p_price[order] / 100.0,
        l_discount=j.p_disc[order] / 100.0,
        l_tax=np.zeros(n, np.float64),
        l_returnflag=np.zeros(n, np.uint8),
        l_linestatus=np.zeros(n, np.uint8),
        n_orders=j.n_build, o_orderkey=j.b_key, o_custkey=j.b_key, o_orderdate=j.b_date,
        n_customer=j.n_build, c_custkey=j.b_key, c_mktsegment=j.b_seg,
    )
    return tables, dict(segment=j.seg_eq, date=date_string(j.date_lt))


def groupby_joined_a_ids(g: GroupByInput) -> np.ndarray:
    """a_id of every B row that survives the three-way join: its c_id names a
    row of C whose category is in the set and whose year is in range, and its
    a_id is an id of A.  Plain numpy; the group-by's input rows."""
    n_c = len(g.c_cat)
    cmask = np.isin(g.c_cat, np.asarray(g.cat_set, dtype=np.uint16)) & (g.c_year >= g.year_lo) & (
        g.c_year <= g.year_hi)
    cid = g.b_c.astype(np.int64)
    inside = (cid >= 0) & (cid < n_c)
    keep = inside.copy()
    keep[inside] = cmask[cid[inside]]
    a = g.b_a[keep]
    return a[np.isin(a, g.a_ids)]


def groupby_as_q18_tables(g: GroupByInput) -> dict:
    """Maps the group-by's count onto run_q18's dense path
    (bespoke_tpch/query_q18.cpp:205-262): one order per id 1..max(A) (dense
    orderkeys, one customer), one lineitem of quantity 1.00 per joined B row
    with l_orderkey = its a_id.  run_q18's sum_qty[orderkey] is then 100 x the
    group's count, and QUANTITY "0" returns every group."""
    a = groupby_joined_a_ids(g)
    n_orders = int(max(int(g.a_ids.max()) if len(g.a_ids) else 1, 1))
    n = len(a)
    return dict(
        n_lineitem=n,
        l_orderkey=np.ascontiguousarray(a, dtype=np.int32),
        l_shipdate=np.full(n, DATE_LO, np.int32),
        l_quantity=np.ones(n, np.float64),
        n_orders=n_orders, o_orderkey=np.arange(1, n_orders + 1, dtype=np.int32),
        o_custkey=np.ones(n_orders, np.int32), o_orderdate=np.full(n_orders, DATE_LO, np.int32),
        n_customer=1, c_custkey=np.ones(1, np.int32), c_mktsegment=np.zeros(1, np.uint8),
    )


def groupby_with_bad_ids(g: GroupByInput) -> GroupByInput:
    """The group-by input with ids no table holds: negative c_ids and c_ids
    past C (rows that join nothing) and a_ids that are not ids of A."""
    g.b_c[::97] = -3
    g.b_c[1::89] = len(g.c_cat) + 5
    g.b_a[2::83] = 10 ** 8
    return g
