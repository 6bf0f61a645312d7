"""Q3 through the C ABI at TPC-H size (1.5M orders, ~6M lineitems) against a
numpy restatement of run_q3 (bespoke_tpch/query_q3.cpp:153-365): result sizes
below and above what one cluster sort holds (131,072 rows; above it the sort
is redone as the pass sequence once the count is read back), rows into
pageable memory (copied after the query) and into mapped pinned memory
(written by the gather kernel), many rows tied on revenue and orderdate (they
come in orderkey order).  Byte-level parity with the reference itself is in
test_dropin_gpu.py."""
import ctypes as C

import numpy as np
import pytest

from bespokeolap_artifacts_b200 import native as N

pytestmark = pytest.mark.gpu

ROW = np.dtype([("rev", "<i8"), ("ok", "<i4"), ("sp", "<i4"), ("od", "<i2"), ("p0", "<i2"), ("p1", "<i4")])


def tables(seed: int, n_orders: int = 1_500_000, n_customer: int = 150_000):
    rng = np.random.default_rng(seed)
    ckey = rng.permutation(np.arange(1, n_customer + 1, dtype=np.int32))
    cseg = rng.integers(0, 3, n_customer).astype(np.uint16)
    okey = (np.arange(n_orders, dtype=np.int64) // 8 * 32 + np.arange(n_orders) % 8 + 1).astype(np.int32)
    ocust = rng.integers(1, n_customer + 30, n_orders).astype(np.int32)  # some name no customer
    odate = np.sort(rng.integers(0, 2405, n_orders)).astype(np.int16)  # orders sorted by date
    oprio = rng.integers(0, 3, n_orders).astype(np.int32)
    lines = rng.integers(1, 8, n_orders)
    lkey = np.repeat(okey, lines)
    n = len(lkey)
    ldate = (np.repeat(odate.astype(np.int32), lines) + rng.integers(1, 2000, n)).clip(max=32767).astype(np.int16)
    ldp = (rng.integers(1, 5, n) * 1000).astype(np.int32)  # coarse prices: many revenue ties
    omap = np.full(int(okey.max()) + 1, -1, np.int32)
    omap[okey] = np.arange(n_orders, dtype=np.int32)
    return dict(ckey=ckey, cseg=cseg, okey=okey, ocust=ocust, odate=odate, oprio=oprio, lkey=lkey, ldate=ldate,
                ldp=ldp, omap=omap)


def q3_oracle(t, date: int, code: int):
    bound = int(t["ckey"].max()) + 1
    inset = np.zeros(bound + 64, bool)
    inset[t["ckey"][t["cseg"] == code]] = True
    oq = (t["odate"] < date) & inset[np.minimum(t["ocust"], bound + 63)]
    lrow = t["omap"][t["lkey"]]
    lpass = (t["ldate"] > date) & oq[lrow]
    no = len(t["okey"])
    rev = np.bincount(lrow[lpass], weights=t["ldp"][lpass].astype(np.float64), minlength=no).astype(np.int64)
    cnt = np.bincount(lrow[lpass], minlength=no)
    rows = np.nonzero(cnt > 0)[0]
    order = np.lexsort((t["okey"][rows], t["odate"][rows], -rev[rows]))
    return rows[order], rev


@pytest.fixture(scope="module")
def q3(engine, torch_cuda):
    torch = torch_cuda
    t = tables(21)
    g = {k: torch.from_numpy(v).cuda() for k, v in t.items()}
    tb = N.TpchQ3Tables()
    tb.c_custkey, tb.c_mktsegment, tb.n_customer = g["ckey"].data_ptr(), g["cseg"].data_ptr(), len(t["ckey"])
    tb.custkey_bound = int(t["ckey"].max()) + 1
    tb.o_orderkey, tb.o_custkey, tb.o_orderdate = g["okey"].data_ptr(), g["ocust"].data_ptr(), g["odate"].data_ptr()
    tb.o_shippriority, tb.n_orders = g["oprio"].data_ptr(), len(t["okey"])
    tb.orderkey_to_row, tb.n_orderkey_map = g["omap"].data_ptr(), len(t["omap"])
    tb.l_orderkey, tb.l_shipdate, tb.l_discounted_price = (g["lkey"].data_ptr(), g["ldate"].data_ptr(),
                                                           g["ldp"].data_ptr())
    tb.n_lineitem = len(t["lkey"])
    return t, g, tb


@pytest.mark.parametrize("date,code", [(100, 1), (600, 0), (1500, 2), (2404, 1)])
@pytest.mark.parametrize("mapped", [False, True])
def test_q3_matches_numpy(engine, q3, date, code, mapped):
    t, _, tb = q3
    want, rev = q3_oracle(t, date, code)
    cap = len(t["okey"])
    n = C.c_int64(-1)
    if mapped:
        buf = C.c_void_p()
        engine.ctx.call("bo_host_alloc_pinned", C.sizeof(N.TpchQ3Row) * cap, C.byref(buf))
        try:
            engine.ctx.call("bo_tpch_q3", C.byref(tb), date, code, C.cast(buf, C.POINTER(N.TpchQ3Row)), cap,
                            C.byref(n))
            got = np.frombuffer((C.c_char * (C.sizeof(N.TpchQ3Row) * cap)).from_address(buf.value), dtype=ROW).copy()
        finally:
            engine.ctx.call("bo_host_free_pinned", buf)
    else:
        out = (N.TpchQ3Row * cap)()
        engine.ctx.call("bo_tpch_q3", C.byref(tb), date, code, out, cap, C.byref(n))
        got = np.frombuffer(out, dtype=ROW)
    assert n.value == len(want)
    got = got[: n.value]
    assert np.array_equal(got["ok"], t["okey"][want])
    assert np.array_equal(got["rev"], rev[want])
    assert np.array_equal(got["od"], t["odate"][want])
    assert np.array_equal(got["sp"], t["oprio"][want])


def test_q3_sizes_cover_both_sort_paths(q3):
    t, _, _ = q3
    sizes = [len(q3_oracle(t, d, c)[0]) for d, c in [(100, 1), (600, 0), (1500, 2), (2404, 1)]]
    assert min(sizes) > 1000 and any(s <= 131_072 for s in sizes) and any(s > 131_072 for s in sizes), sizes


def test_q3_rows_past_max_rows_are_not_written(engine, q3):
    """max_rows below the result size: the count is the full size, only the
    first max_rows rows are written (the rest of the buffer is untouched)."""
    t, _, tb = q3
    want, rev = q3_oracle(t, 600, 0)
    buf = C.c_void_p()
    cap = 1001  # odd: the last block's rows end mid 16-byte word
    engine.ctx.call("bo_host_alloc_pinned", C.sizeof(N.TpchQ3Row) * (cap + 8), C.byref(buf))
    try:
        raw = (C.c_char * (C.sizeof(N.TpchQ3Row) * (cap + 8))).from_address(buf.value)
        C.memset(buf.value, 0x5A, C.sizeof(raw))
        n = C.c_int64(-1)
        engine.ctx.call("bo_tpch_q3", C.byref(tb), 600, 0, C.cast(buf, C.POINTER(N.TpchQ3Row)), cap, C.byref(n))
        got = np.frombuffer(raw, dtype=ROW).copy()
    finally:
        engine.ctx.call("bo_host_free_pinned", buf)
    assert n.value == len(want) > cap
    assert np.array_equal(got["ok"][:cap], t["okey"][want[:cap]])
    assert np.array_equal(got["rev"][:cap], rev[want[:cap]])
    assert (got.view(np.uint8)[cap * ROW.itemsize:] == 0x5A).all()
