"""Q4 through the C ABI at 1.5M orders / ~6M lineitems against a numpy
restatement of run_q4 (bespoke_tpch/query_q4.cpp:172-355): lineitems sorted
by orderkey (the range walk) and shuffled (the range walk that checks each
lineitem's key), commit / receipt offsets on both sides of zero (the
unsigned 16-bit comparison of q4_is_late, :71-73).  Byte-level parity with
the reference itself is in test_dropin_gpu.py."""
import ctypes as C

import numpy as np
import pytest

from bespokeolap_artifacts_b200 import native as N

pytestmark = pytest.mark.gpu


def data(n_orders: int, seed: int, shuffle: bool):
    rng = np.random.default_rng(seed)
    okey = (np.arange(n_orders, dtype=np.int64) // 8 * 32 + np.arange(n_orders) % 8 + 1).astype(np.int32)
    odate = rng.integers(-30, 2405, n_orders).astype(np.int16)
    prio = rng.integers(0, 5, n_orders).astype(np.uint16)
    order = np.argsort(odate, kind="stable")
    okey, odate, prio = okey[order], odate[order], prio[order]
    lines = rng.integers(0, 8, n_orders)  # some orders without lineitems
    lkey = np.repeat(np.sort(okey), lines[np.argsort(okey)])
    n = len(lkey)
    if shuffle:
        lkey = lkey[rng.permutation(n)]
    commit = rng.integers(-40, 2500, n)
    receipt = commit + rng.integers(-45, 15, n)
    cr = ((receipt.astype(np.int64) & 0xFFFF) << 16) | (commit.astype(np.int64) & 0xFFFF)
    omap = np.full(int(okey.max()) + 1, -1, np.int32)
    omap[okey] = np.arange(n_orders, dtype=np.int32)
    return dict(okey=okey, odate=odate, prio=prio, lkey=lkey, cr=cr.astype(np.uint32), omap=omap, sorted=not shuffle)


def restate(d, start, end, n_prio=5):
    cr = d["cr"]
    late = (cr & 0xFFFF) < (cr >> 16)  # unsigned 16-bit offsets
    late_keys = np.unique(d["lkey"][late])
    sel = (d["odate"] >= start) & (d["odate"] < end) & np.isin(d["okey"], late_keys)
    return np.bincount(d["prio"][sel], minlength=n_prio).tolist()


@pytest.mark.parametrize("shuffle", [False, True])
def test_q4_matches_numpy(engine, torch_cuda, shuffle):
    torch = torch_cuda
    d = data(1_500_000, 21 + shuffle, shuffle)
    g = {k: torch.from_numpy(v.view(np.int16) if v.dtype == np.uint16 else
                             (v.view(np.int32) if v.dtype == np.uint32 else v)).cuda()
         for k, v in d.items() if isinstance(v, np.ndarray)}
    n_orders = len(d["okey"])
    begin = torch.empty(n_orders, dtype=torch.int32, device="cuda")
    end_ = torch.empty(n_orders, dtype=torch.int32, device="cuda")
    engine.ctx.call("bo_tpch_order_ranges", C.c_void_p(g["lkey"].data_ptr()), len(d["lkey"]),
                    C.c_void_p(g["omap"].data_ptr()), len(d["omap"]), n_orders, C.c_void_p(begin.data_ptr()),
                    C.c_void_p(end_.data_ptr()))
    t = N.TpchQ4Tables()
    t.o_orderkey, t.o_orderdate, t.o_orderpriority = g["okey"].data_ptr(), g["odate"].data_ptr(), g["prio"].data_ptr()
    t.o_li_begin, t.o_li_end, t.n_orders = begin.data_ptr(), end_.data_ptr(), n_orders
    t.l_orderkey, t.l_commit_receipt, t.n_lineitem = g["lkey"].data_ptr(), g["cr"].data_ptr(), len(d["lkey"])
    t.lineitem_orderkey_sorted, t.n_priorities = int(d["sorted"]), 5
    for start, end in [(547, 639), (-30, 60), (2300, 2500), (3000, 3090), (400, 400)]:
        counts = (C.c_int64 * 5)()
        engine.ctx.call("bo_tpch_q4", C.byref(t), start, end, counts)
        assert list(counts) == restate(d, start, end), (start, end)


def test_q4_arguments(engine):
    t = N.TpchQ4Tables()
    t.n_orders, t.n_priorities = 4, 5
    counts = (C.c_int64 * 5)()
    with pytest.raises(N.BoError):
        engine.ctx.call("bo_tpch_q4", C.byref(t), 0, 10, counts)  # null columns
    t.n_orders, t.n_priorities = 0, -1
    with pytest.raises(N.BoError):
        engine.ctx.call("bo_tpch_q4", C.byref(t), 0, 10, counts)  # negative priority count
    t.n_priorities = 5
    engine.ctx.call("bo_tpch_q4", C.byref(t), 0, 10, counts)
    assert list(counts) == [0] * 5
