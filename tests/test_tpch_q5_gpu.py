"""Q5 through the C ABI at 1.5M orders / ~6M lineitems against a numpy
restatement of run_q5 (bespoke_tpch/query_q5.cpp:197-540): lineitems sorted
by orderkey and shuffled, customer and supplier nations including -1 (no
customer / supplier row) and nations outside the region.  Byte-level parity
with the reference itself is in test_dropin_gpu.py."""
import ctypes as C

import numpy as np
import pytest

from bespokeolap_artifacts_b200 import native as N

pytestmark = pytest.mark.gpu

N_NATIONS = 25


def data(n_orders: int, seed: int, shuffle: bool):
    rng = np.random.default_rng(seed)
    okey = (np.arange(n_orders, dtype=np.int64) // 8 * 32 + np.arange(n_orders) % 8 + 1).astype(np.int32)
    odate = rng.integers(0, 2405, n_orders).astype(np.int16)
    cnat = rng.integers(-1, N_NATIONS, n_orders).astype(np.int16)
    order = np.argsort(odate, kind="stable")
    okey, odate, cnat = okey[order], odate[order], cnat[order]
    lines = rng.integers(0, 8, n_orders)
    lkey = np.repeat(np.sort(okey), lines[np.argsort(okey)])
    n = len(lkey)
    if shuffle:
        lkey = lkey[rng.permutation(n)]
    snat = rng.integers(-1, N_NATIONS, n).astype(np.int16)
    price = rng.integers(-1_000, 10_500_000, n).astype(np.int32)
    omap = np.full(int(okey.max()) + 1, -1, np.int32)
    omap[okey] = np.arange(n_orders, dtype=np.int32)
    return dict(okey=okey, odate=odate, cnat=cnat, lkey=lkey, snat=snat, price=price, omap=omap, sorted=not shuffle)


def restate(d, in_region, start, end):
    row = d["omap"][d["lkey"]]  # every lineitem's order row (all keys have one)
    cn = d["cnat"][row]
    ok = (d["odate"][row] >= start) & (d["odate"][row] < end) & (cn >= 0)
    ok &= in_region[np.where(cn >= 0, cn, 0)].astype(bool) & (d["snat"] == cn)
    price = d["price"].astype(np.int64)
    return [int(price[ok & (cn == k)].sum()) for k in range(N_NATIONS)]


@pytest.mark.parametrize("shuffle", [False, True])
def test_q5_matches_numpy(engine, torch_cuda, shuffle):
    torch = torch_cuda
    d = data(1_500_000, 50 + shuffle, shuffle)
    g = {k: torch.from_numpy(v).cuda() for k, v in d.items() if isinstance(v, np.ndarray)}
    n_orders = len(d["okey"])
    begin = torch.empty(n_orders, dtype=torch.int32, device="cuda")
    end_ = torch.empty(n_orders, dtype=torch.int32, device="cuda")
    engine.ctx.call("bo_tpch_order_ranges", C.c_void_p(g["lkey"].data_ptr()), len(d["lkey"]),
                    C.c_void_p(g["omap"].data_ptr()), len(d["omap"]), n_orders, C.c_void_p(begin.data_ptr()),
                    C.c_void_p(end_.data_ptr()))
    t = N.TpchQ5Tables()
    t.o_orderkey, t.o_orderdate, t.o_cust_nation = g["okey"].data_ptr(), g["odate"].data_ptr(), g["cnat"].data_ptr()
    t.o_li_begin, t.o_li_end, t.n_orders = begin.data_ptr(), end_.data_ptr(), n_orders
    t.l_orderkey, t.l_supp_nation, t.l_discounted_price = g["lkey"].data_ptr(), g["snat"].data_ptr(), g["price"].data_ptr()
    t.n_lineitem, t.lineitem_orderkey_sorted, t.n_nations = len(d["lkey"]), int(d["sorted"]), N_NATIONS
    rng = np.random.default_rng(5)
    for start, end in [(731, 1096), (0, 366), (2300, 2665), (3000, 3365)]:
        in_region = (rng.random(N_NATIONS) < 0.3).astype(np.uint8)
        rev = (C.c_int64 * N_NATIONS)()
        engine.ctx.call("bo_tpch_q5", C.byref(t), in_region.tobytes(), start, end, rev)
        assert list(rev) == restate(d, in_region, start, end), (start, end)


def test_q5_arguments(engine):
    t = N.TpchQ5Tables()
    t.n_orders, t.n_nations = 4, 25
    rev = (C.c_int64 * 25)()
    with pytest.raises(N.BoError):
        engine.ctx.call("bo_tpch_q5", C.byref(t), bytes(25), 0, 10, rev)  # null columns
    t.n_orders, t.n_nations = 0, 40000
    with pytest.raises(N.BoError):
        engine.ctx.call("bo_tpch_q5", C.byref(t), bytes(40000), 0, 10, rev)  # nation keys beyond int16
