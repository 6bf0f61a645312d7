"""Q14 through the C ABI at 6M lineitems against a numpy restatement of
run_q14's sums (bespoke_tpch/query_q14.cpp:176-352): lineitems shipped in
the month whose partkey has a part row, all and promo-typed; partkeys that
are negative, beyond the part keys or without a part row are skipped.
Byte-level parity of the formatted result with the reference is in
test_dropin_gpu.py."""
import ctypes as C

import numpy as np
import pytest

from bespokeolap_artifacts_b200 import native as N

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def q14_data(torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(14)
    n = 6_000_003  # a ragged tail
    ship = rng.integers(-20, 2530, n).astype(np.int16)
    pkey = rng.integers(-5, 210_000, n).astype(np.int32)
    price = rng.integers(-1_000, 10_500_000, n).astype(np.int32)
    promo = rng.integers(-1, 2, 200_001).astype(np.int8)  # keys 0..200000; -1 = no part row
    d = dict(ship=ship, pkey=pkey, price=price, promo=promo)
    g = {k: torch.from_numpy(v).cuda() for k, v in d.items()}
    return d, g


@pytest.mark.parametrize("window", [(1338, 1368), (-20, 11), (2500, 2531), (0, 0), (3000, 3030)])
def test_q14_matches_numpy(engine, q14_data, window):
    d, g = q14_data
    start, end = window
    t = N.TpchQ14Tables()
    t.l_shipdate, t.l_partkey, t.l_discounted_price = g["ship"].data_ptr(), g["pkey"].data_ptr(), g["price"].data_ptr()
    t.n_lineitem, t.p_promo_by_key, t.n_promo_map = len(d["ship"]), g["promo"].data_ptr(), len(d["promo"])
    sums = (C.c_int64 * 2)()
    engine.ctx.call("bo_tpch_q14", C.byref(t), start, end, sums)
    k = d["pkey"].astype(np.int64)
    ok = (d["ship"] >= start) & (d["ship"] < end) & (k >= 0) & (k < len(d["promo"]))
    flag = d["promo"][np.where(ok, k, 0)]
    ok &= flag >= 0
    price = d["price"].astype(np.int64)
    assert list(sums) == [int(price[ok & (flag == 1)].sum()), int(price[ok].sum())]


def test_q14_arguments(engine, q14_data):
    d, g = q14_data
    t = N.TpchQ14Tables()
    t.n_lineitem = 8
    sums = (C.c_int64 * 2)()
    with pytest.raises(N.BoError):
        engine.ctx.call("bo_tpch_q14", C.byref(t), 0, 30, sums)  # null columns
    t.l_shipdate, t.l_partkey, t.l_discounted_price = g["ship"].data_ptr() + 2, g["pkey"].data_ptr(), g["price"].data_ptr()
    with pytest.raises(N.BoError):
        engine.ctx.call("bo_tpch_q14", C.byref(t), 0, 30, sums)  # misaligned shipdates
