"""Q8 through the C ABI at ~6M lineitems against a numpy restatement of
run_q8 (bespoke_tpch/query_q8.cpp:122-380): lineitems of one part type whose
order falls in 1995-1996 and was placed by a customer of the region, volume
per order year in total and for suppliers of the target nation; customer
keys repeated with different nations (any of them in the region marks the
key), keys outside every table.  Byte-level parity of the formatted result
with the reference is in test_dropin_gpu.py."""
import ctypes as C

import numpy as np
import pytest

from bespokeolap_artifacts_b200 import native as N

pytestmark = pytest.mark.gpu

START, LAST, YEAR2 = 1096, 1826, 1461  # 1995-01-01, 1996-12-31, 1996-01-01 as offsets from 1992-01-01


@pytest.fixture(scope="module")
def q8_data(torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(8)
    n_orders, n, n_cust, n_part = 1_500_000, 6_000_007, 150_000, 200_000
    okeys = rng.choice(np.arange(1, n_orders * 4 + 1), n_orders, replace=False).astype(np.int32)
    omap = np.full(n_orders * 4 + 8, -1, np.int32)
    omap[okeys] = np.arange(n_orders, dtype=np.int32)
    ocust = rng.integers(-3, n_cust + 50, n_orders).astype(np.int32)
    odate = rng.integers(0, 2560, n_orders).astype(np.int16)
    ckey = np.concatenate([np.arange(1, n_cust + 1), rng.integers(1, n_cust + 1, 500)]).astype(np.int32)
    cnat = rng.integers(-1, 27, len(ckey)).astype(np.int32)
    pkey = np.concatenate([np.arange(1, n_part + 1), [-4, 7]]).astype(np.int32)
    ptype = rng.integers(0, 150, len(pkey)).astype(np.uint16)
    lpk = rng.integers(-2, n_part + 300, n).astype(np.int32)
    lsk = rng.integers(-1, 10_010, n).astype(np.int32)
    lok = okeys[rng.integers(0, n_orders, n)]
    lok[rng.integers(0, n, 1000)] = rng.integers(-5, n_orders * 4 + 100, 1000)
    price = rng.integers(90_000, 10_500_000, n).astype(np.int32)
    disc = rng.integers(0, 11, n).astype(np.uint8)
    d = dict(omap=omap, ocust=ocust, odate=odate, ckey=ckey, cnat=cnat, pkey=pkey, ptype=ptype, lpk=lpk, lsk=lsk,
             lok=lok, price=price, disc=disc)
    g = {k: torch.from_numpy(v.view(np.int16) if v.dtype == np.uint16 else v).cuda() for k, v in d.items()}
    return d, g


def restate(d, in_region, supp, type_code):
    max_c, max_p = int(d["ckey"].max()), int(d["pkey"].max())
    cust_ok = np.zeros(max_c + 1, bool)
    ok_c = (d["cnat"] >= 0) & (d["cnat"] < len(in_region))
    ok_c[ok_c] = in_region[d["cnat"][ok_c]].astype(bool)
    cust_ok[d["ckey"][ok_c]] = True
    part_ok = np.zeros(max_p + 1, bool)
    sel = (d["pkey"] >= 0) & (d["ptype"] == type_code)
    part_ok[d["pkey"][sel]] = True
    pk = d["lpk"].astype(np.int64)
    ok = (pk >= 0) & (pk <= max_p)
    ok[ok] = part_ok[pk[ok]]
    k = d["lok"].astype(np.int64)
    ok &= (k >= 0) & (k < len(d["omap"]))
    row = np.where(ok, d["omap"][np.where(ok, k, 0)], -1)
    ok &= row >= 0
    r = np.where(ok, row, 0)
    date = d["odate"][r].astype(np.int64)
    ok &= (date >= START) & (date <= LAST)
    ck = d["ocust"][r].astype(np.int64)
    ok &= (ck >= 0) & (ck <= max_c)
    ok[ok] = cust_ok[ck[ok]]
    vol = d["price"].astype(np.int64) * (100 - d["disc"].astype(np.int64))
    sk = d["lsk"].astype(np.int64)
    tgt = (sk >= 0) & (sk < len(supp))
    tgt[tgt] = supp[sk[tgt]].astype(bool)
    y = date >= YEAR2
    return [int(vol[ok & tgt & ~y].sum()), int(vol[ok & tgt & y].sum()), int(vol[ok & ~y].sum()),
            int(vol[ok & y].sum())]


@pytest.mark.parametrize("type_code", [7, 0, 149, 200])
def test_q8_matches_numpy(engine, q8_data, type_code):
    d, g = q8_data
    rng = np.random.default_rng(type_code)
    in_region = (rng.random(25) < 0.2).astype(np.uint8)
    supp = (rng.random(10_000) < 0.04).astype(np.uint8)
    t = N.TpchQ8Tables()
    t.l_partkey, t.l_suppkey, t.l_orderkey = g["lpk"].data_ptr(), g["lsk"].data_ptr(), g["lok"].data_ptr()
    t.l_extendedprice, t.l_discount, t.n_lineitem = g["price"].data_ptr(), g["disc"].data_ptr(), len(d["lpk"])
    t.orderkey_to_row, t.n_orderkey_map = g["omap"].data_ptr(), len(d["omap"])
    t.o_custkey, t.o_orderdate, t.n_orders = g["ocust"].data_ptr(), g["odate"].data_ptr(), len(d["ocust"])
    t.c_custkey, t.c_nationkey, t.n_customer = g["ckey"].data_ptr(), g["cnat"].data_ptr(), len(d["ckey"])
    t.max_custkey, t.max_partkey = int(d["ckey"].max()), int(d["pkey"].max())
    t.p_partkey, t.p_type, t.n_part = g["pkey"].data_ptr(), g["ptype"].data_ptr(), len(d["pkey"])
    sums = (C.c_int64 * 4)()
    engine.ctx.call("bo_tpch_q8", C.byref(t), in_region.tobytes(), 25, supp.tobytes(), len(supp), type_code, START,
                    LAST, YEAR2, sums)
    assert list(sums) == restate(d, in_region, supp, type_code)


def test_q8_arguments(engine):
    t = N.TpchQ8Tables()
    t.n_lineitem, t.max_partkey, t.max_custkey = 8, 5, 5
    sums = (C.c_int64 * 4)()
    with pytest.raises(N.BoError):
        engine.ctx.call("bo_tpch_q8", C.byref(t), bytes(25), 25, bytes(4), 4, 0, START, LAST, YEAR2, sums)
