"""Q7 through the C ABI at ~6M lineitems against a numpy restatement of
run_q7 (bespoke_tpch/query_q7.cpp:140-435): lineitems shipped in the
two-year window (both ends included) by tagged suppliers, joined to their
order's customer nation, summed by (supplier nation, customer nation,
year); two nations and one nation twice; suppkeys outside the tag table,
orderkeys without an order.  Byte-level parity with the reference is in
test_dropin_gpu.py."""
import ctypes as C

import numpy as np
import pytest

from bespokeolap_artifacts_b200 import native as N

pytestmark = pytest.mark.gpu

START, LAST, YEAR2 = 1096, 1826, 1461  # 1995-01-01, 1996-12-31, 1996-01-01 as offsets from 1992-01-01


@pytest.fixture(scope="module")
def q7_data(torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(7)
    n_orders, n = 1_500_000, 6_000_001
    omap = np.full(n_orders * 4 + 8, -1, np.int32)
    okeys = rng.choice(np.arange(1, n_orders * 4 + 1), n_orders, replace=False).astype(np.int32)
    omap[okeys] = np.arange(n_orders, dtype=np.int32)
    cnat = rng.integers(-1, 25, n_orders).astype(np.int16)
    lok = okeys[rng.integers(0, n_orders, n)]
    lok[rng.integers(0, n, 1000)] = rng.integers(-5, n_orders * 4 + 100, 1000)
    ship = rng.integers(0, 2560, n).astype(np.int16)
    sk = rng.integers(-2, 10_040, n).astype(np.int32)
    price = rng.integers(-1_000, 10_500_000, n).astype(np.int32)
    d = dict(omap=omap, cnat=cnat, lok=lok, ship=ship, sk=sk, price=price)
    g = {k: torch.from_numpy(v).cuda() for k, v in d.items()}
    return d, g


def restate(d, tag, n1, n2):
    same = n1 == n2
    ship = d["ship"].astype(np.int64)
    ok = (ship >= START) & (ship <= LAST)
    sk = d["sk"].astype(np.int64)
    ok &= (sk >= 0) & (sk < len(tag))
    supp = np.where(ok, tag[np.where(ok, sk, 0)], -1).astype(np.int64)
    ok &= supp >= 0
    k = d["lok"].astype(np.int64)
    ok &= (k >= 0) & (k < len(d["omap"]))
    row = np.where(ok, d["omap"][np.where(ok, k, 0)], -1)
    ok &= row >= 0
    cn = np.where(ok, d["cnat"][np.where(ok, row, 0)], -9).astype(np.int64)
    cust = np.where(cn == n1, 0, np.where((~np.bool_(same)) & (cn == n2), 1, -1))
    ok &= cust >= 0
    ok &= (supp == 0) & (cust == 0) if same else (supp != cust)
    idx = supp * 4 + cust * 2 + (ship >= YEAR2)
    price = d["price"].astype(np.int64)
    return [int(price[ok & (idx == i)].sum()) for i in range(8)]


@pytest.mark.parametrize("nations", [(3, 11), (11, 3), (5, 5), (0, 24)])
def test_q7_matches_numpy(engine, q7_data, nations):
    d, g = q7_data
    rng = np.random.default_rng(nations[0] * 31 + nations[1])
    s_nation = rng.integers(0, 25, 10_000)
    n1, n2 = nations
    tag = np.full(10_000, -1, np.int8)
    tag[s_nation == n1] = 0
    if n1 != n2:
        tag[s_nation == n2] = 1
    t = N.TpchQ7Tables()
    t.l_shipdate, t.l_suppkey, t.l_orderkey = g["ship"].data_ptr(), g["sk"].data_ptr(), g["lok"].data_ptr()
    t.l_discounted_price, t.n_lineitem = g["price"].data_ptr(), len(d["ship"])
    t.orderkey_to_row, t.n_orderkey_map = g["omap"].data_ptr(), len(d["omap"])
    t.o_cust_nation, t.n_orders = g["cnat"].data_ptr(), len(d["cnat"])
    rev = (C.c_int64 * 8)()
    engine.ctx.call("bo_tpch_q7", C.byref(t), tag.tobytes(), len(tag), n1, n2, START, LAST, YEAR2, rev)
    assert list(rev) == restate(d, tag, n1, n2)


def test_q7_arguments(engine, q7_data):
    d, g = q7_data
    t = N.TpchQ7Tables()
    t.n_lineitem = 8
    rev = (C.c_int64 * 8)()
    with pytest.raises(N.BoError):
        engine.ctx.call("bo_tpch_q7", C.byref(t), bytes(4), 4, 0, 1, START, LAST, YEAR2, rev)  # null columns
