"""Q15 through the C ABI at ~6M lineitems against a numpy restatement of
run_q15's per-supplier totals (bespoke_tpch/query_q15.cpp:215-534): the
quarter's lineitems summed per suppkey (keys above 4096 go through the
global totals, negative and out-of-range keys are not summed), and the count
of lineitems in the window.  Byte-level parity of the formatted result with
the reference is in test_dropin_gpu.py."""
import ctypes as C

import numpy as np
import pytest

from bespokeolap_artifacts_b200 import native as N

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def q15_data(torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(15)
    n = 6_000_005
    ship = rng.integers(-10, 2560, n).astype(np.int16)
    sk = rng.integers(-3, 10_100, n).astype(np.int32)
    price = rng.integers(-1_000, 10_500_000, n).astype(np.int32)
    d = dict(ship=ship, sk=sk, price=price)
    return d, {k: torch.from_numpy(v).cuda() for k, v in d.items()}


@pytest.mark.parametrize("window", [(1461, 1552), (0, 90), (2500, 2591), (3000, 3091)])
@pytest.mark.parametrize("n_supp", [10_001, 25, 1])
def test_q15_matches_numpy(engine, q15_data, window, n_supp):
    d, g = q15_data
    start, end = window
    t = N.TpchQ15Tables()
    t.l_shipdate, t.l_suppkey, t.l_discounted_price = g["ship"].data_ptr(), g["sk"].data_ptr(), g["price"].data_ptr()
    t.n_lineitem = len(d["ship"])
    rev = (C.c_int64 * n_supp)()
    shipped = C.c_int64()
    engine.ctx.call("bo_tpch_q15", C.byref(t), n_supp, start, end, rev, C.byref(shipped))
    s = d["ship"].astype(np.int64)
    win = (s >= start) & (s < end)
    k = d["sk"].astype(np.int64)
    ok = win & (k >= 0) & (k < n_supp)
    keys = [i for i in list(range(30)) + list(range(4090, 4110)) if i < n_supp]  # shared and global totals
    want = [int(d["price"][ok & (k == i)].astype(np.int64).sum()) for i in keys]
    assert [rev[i] for i in keys] == want
    assert sum(rev) == int(d["price"][ok].astype(np.int64).sum())
    assert shipped.value == int(win.sum())
