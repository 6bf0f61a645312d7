"""Q10, Q18 and the per-order lineitem ranges through the C ABI at sizes the
drop-in files do not reach (millions of lineitems), against numpy
restatements of run_q10 (bespoke_tpch/query_q10.cpp:375-585), run_q18
(bespoke_tpch/query_q18.cpp:183-455) and the builder's ranges
(bespoke_tpch/builder_impl.cpp:930-990); plus the entry points' error
contract.  Byte-level parity with the reference itself is in
test_dropin_gpu.py."""
import ctypes as C

import numpy as np
import pytest

from bespokeolap_artifacts_b200 import native as N

pytestmark = pytest.mark.gpu


def tables(n_orders: int, seed: int, shuffle: bool = False, n_customer: int = 150_000):
    rng = np.random.default_rng(seed)
    okey = (np.arange(n_orders, dtype=np.int64) // 8 * 32 + np.arange(n_orders) % 8 + 1).astype(np.int32)
    ocust = rng.integers(0, n_customer + 20, n_orders).astype(np.int32)  # some without a customer
    odate = rng.integers(0, 2405, n_orders).astype(np.int16)
    ototal = rng.integers(100_000, 50_000_000, n_orders).astype(np.int32)
    order = np.argsort(odate, kind="stable")
    okey, ocust, odate, ototal = okey[order], ocust[order], odate[order], ototal[order]
    lines = rng.integers(1, 8, n_orders)
    lkey = np.repeat(np.sort(okey), lines)
    n = len(lkey)
    if shuffle:
        lkey = lkey[rng.permutation(n)]
    lqty = (rng.integers(1, 51, n) * 100).astype(np.int16)
    lcode = rng.integers(0, 6, n).astype(np.uint8)  # returnflag (3) x linestatus (2)
    ldp = rng.integers(90_000, 10_500_000, n).astype(np.int32)
    ckey = rng.permutation(np.arange(1, n_customer + 1, dtype=np.int32) * 2)[: n_customer]
    cmap = np.full(int(ckey.max()) + 1, -1, np.int32)
    cmap[ckey] = np.arange(n_customer, dtype=np.int32)
    cnation = rng.integers(-1, 27, n_customer).astype(np.int32)
    omap = np.full(int(okey.max()) + 1, -1, np.int32)
    omap[okey] = np.arange(n_orders, dtype=np.int32)
    return dict(okey=okey, ocust=ocust, odate=odate, ototal=ototal, lkey=lkey, lqty=lqty, lcode=lcode, ldp=ldp,
                cmap=cmap, cnation=cnation, omap=omap, sorted=not shuffle)


def dev(torch, d):
    return {k: (torch.from_numpy(v).cuda() if isinstance(v, np.ndarray) else v) for k, v in d.items()}


def ranges(engine, torch, g, n_orders):
    begin = torch.empty(n_orders, dtype=torch.int32, device="cuda")
    end = torch.empty(n_orders, dtype=torch.int32, device="cuda")
    engine.ctx.call("bo_tpch_order_ranges", C.c_void_p(g["lkey"].data_ptr()), g["lkey"].numel(),
                    C.c_void_p(g["omap"].data_ptr()), g["omap"].numel(), n_orders, C.c_void_p(begin.data_ptr()),
                    C.c_void_p(end.data_ptr()))
    torch.cuda.synchronize()
    return begin, end


@pytest.mark.parametrize("shuffle", [False, True])
def test_order_ranges(engine, torch_cuda, shuffle):
    torch = torch_cuda
    t = tables(200_000, 1, shuffle)
    g = dev(torch, t)
    begin, end = ranges(engine, torch, g, len(t["okey"]))
    rows = t["omap"][t["lkey"]]
    idx = np.arange(len(rows), dtype=np.int64)
    want_b = np.full(len(t["okey"]), 0xFFFFFFFF, np.int64)
    want_e = np.zeros(len(t["okey"]), np.int64)
    np.minimum.at(want_b, rows, idx)
    np.maximum.at(want_e, rows, idx + 1)
    assert np.array_equal(begin.cpu().numpy().view(np.uint32).astype(np.int64), want_b)
    assert np.array_equal(end.cpu().numpy().view(np.uint32).astype(np.int64), want_e)


def q18_oracle(t, thr):
    """Non-dense path (:292-434): every orders row whose orderkey's quantity
    sum exceeds thr and whose customer has a row."""
    sums = np.zeros(max(int(t["okey"].max()), int(t["lkey"].max())) + 1, np.int64)
    np.add.at(sums, t["lkey"], t["lqty"].astype(np.int64))
    s = sums[t["okey"]]
    c = t["ocust"]
    crow = np.where(c < len(t["cmap"]), t["cmap"][np.minimum(c, len(t["cmap"]) - 1)], -1)
    keep = (s > thr) & (crow >= 0)
    rows = np.nonzero(keep)[0]
    order = np.lexsort((t["okey"][rows], t["odate"][rows], -t["ototal"][rows].astype(np.int64)))
    rows = rows[order]
    return s[rows], c[rows], crow[rows], t["okey"][rows], t["ototal"][rows], t["odate"][rows]


@pytest.mark.parametrize("thr", [25_000, 30_000, 0])
@pytest.mark.parametrize("mapped", [False, True])
def test_q18_matches_numpy(engine, torch_cuda, thr, mapped):
    """Rows into pageable memory (copied) and into mapped pinned memory
    (written by the gather kernel); threshold 0 keeps more orders than one
    cluster sort holds (the query reruns with the count read back)."""
    torch = torch_cuda
    t = tables(1_500_000, 2)
    g = dev(torch, t)
    tb = N.TpchQ18Tables()
    tb.o_orderkey, tb.o_custkey = g["okey"].data_ptr(), g["ocust"].data_ptr()
    tb.o_orderdate, tb.o_totalprice = g["odate"].data_ptr(), g["ototal"].data_ptr()
    tb.n_orders = len(t["okey"])
    tb.l_orderkey, tb.l_quantity, tb.n_lineitem = g["lkey"].data_ptr(), g["lqty"].data_ptr(), len(t["lkey"])
    tb.custkey_to_row, tb.n_custkey_map = g["cmap"].data_ptr(), len(t["cmap"])
    tb.n_customer = 150_000
    tb.orderkey_bound = max(int(t["okey"].max()), int(t["lkey"].max())) + 1
    cap = len(t["okey"])
    n = C.c_int64()
    row_t = np.dtype([("sum", "<i8"), ("cust", "<i4"), ("crow", "<i4"), ("okey", "<i4"), ("total", "<i4"),
                      ("date", "<i2"), ("p0", "<i2"), ("p1", "<i4")])
    if mapped:
        buf = C.c_void_p()
        engine.ctx.call("bo_host_alloc_pinned", C.sizeof(N.TpchQ18Row) * cap, C.byref(buf))
        try:
            engine.ctx.call("bo_tpch_q18", C.byref(tb), thr, C.cast(buf, C.POINTER(N.TpchQ18Row)), cap, C.byref(n))
            got = np.frombuffer((C.c_char * (C.sizeof(N.TpchQ18Row) * cap)).from_address(buf.value),
                                dtype=row_t).copy()
        finally:
            engine.ctx.call("bo_host_free_pinned", buf)
    else:
        out = (N.TpchQ18Row * cap)()
        engine.ctx.call("bo_tpch_q18", C.byref(tb), thr, out, cap, C.byref(n))
        got = np.frombuffer(out, dtype=row_t)
    want = q18_oracle(t, thr)
    assert n.value == len(want[0]) and n.value > 0
    if thr == 0:
        assert n.value > 131_072
    got = got[: n.value]
    for name, w in zip(("sum", "cust", "crow", "okey", "total", "date"), want):
        assert np.array_equal(got[name], w), name


def q10_oracle(t, start, end, glo, gcount, nation_bound):
    n_map = len(t["cmap"])
    rows = np.nonzero((t["odate"] >= start) & (t["odate"] < end) & (t["ocust"] >= 0) & (t["ocust"] < n_map))[0]
    lrow = t["omap"][t["lkey"]]
    ok = ((t["lcode"].astype(np.int64) - glo) >= 0) & ((t["lcode"].astype(np.int64) - glo) < gcount)
    rev = np.zeros(len(t["okey"]), np.int64)
    np.add.at(rev, lrow[ok], t["ldp"][ok].astype(np.int64))
    rows = rows[rev[rows] != 0]
    cust = np.zeros(n_map, np.int64)
    hit = np.zeros(n_map, bool)
    np.add.at(cust, t["ocust"][rows], rev[rows])
    hit[t["ocust"][rows]] = True
    ck = np.nonzero(hit)[0]
    crow = t["cmap"][ck]
    ck, crow = ck[crow >= 0], crow[crow >= 0]
    nk = t["cnation"][crow]
    sel = (nk >= 0) & (nk < nation_bound)
    ck, crow, nk = ck[sel], crow[sel], nk[sel]
    r = cust[ck]
    order = np.lexsort((ck, ~r.view(np.uint64)))
    return r[order], ck[order], crow[order], nk[order]


@pytest.mark.parametrize("shuffle", [False, True])
def test_q10_matches_numpy(engine, torch_cuda, shuffle):
    torch = torch_cuda
    t = tables(1_500_000, 3, shuffle)
    g = dev(torch, t)
    no = len(t["okey"])
    begin, end = ranges(engine, torch, g, no)
    tb = N.TpchQ10Tables()
    tb.o_orderkey, tb.o_custkey, tb.o_orderdate = g["okey"].data_ptr(), g["ocust"].data_ptr(), g["odate"].data_ptr()
    tb.o_li_begin, tb.o_li_end, tb.n_orders = begin.data_ptr(), end.data_ptr(), no
    tb.l_orderkey, tb.l_returnflag_linestatus = g["lkey"].data_ptr(), g["lcode"].data_ptr()
    tb.l_discounted_price, tb.n_lineitem = g["ldp"].data_ptr(), len(t["lkey"])
    tb.lineitem_orderkey_sorted = 1 if t["sorted"] else 0
    tb.nation_bound = 25
    tb.custkey_to_row, tb.n_custkey_map = g["cmap"].data_ptr(), len(t["cmap"])
    tb.c_nationkey, tb.n_customer = g["cnation"].data_ptr(), len(t["cnation"])
    # Every other pass also gathers the customers' string ranges and balances
    # (random offsets per column, as the host's string columns store them).
    nc = len(t["cnation"])
    rng = np.random.default_rng(5)
    offs = [np.concatenate([[0], np.cumsum(rng.integers(0, 90, size=nc))]).astype(np.uint32) for _ in range(4)]
    acct = rng.integers(-99_999, 999_999, size=nc).astype(np.int32)
    offs_d = [torch.from_numpy(o).cuda() for o in offs]
    acct_d = torch.from_numpy(acct).cuda()
    row_t = np.dtype([("rev", "<i8"), ("cust", "<i4"), ("crow", "<i4"), ("nk", "<i4"), ("acct", "<i4"),
                      ("b0", "<u4"), ("l0", "<u4"), ("b1", "<u4"), ("l1", "<u4"), ("b2", "<u4"), ("l2", "<u4"),
                      ("b3", "<u4"), ("l3", "<u4")])
    assert row_t.itemsize == C.sizeof(N.TpchQ10Row)
    for pass_no, (start, end_) in enumerate([(640, 730), (0, 2405), (100, 100), (0, 2405)]):
        strings = pass_no % 2 == 1
        tb.c_name_offsets, tb.c_address_offsets, tb.c_phone_offsets, tb.c_comment_offsets = (
            [o.data_ptr() for o in offs_d] if strings else [None] * 4)
        tb.c_acctbal = acct_d.data_ptr() if strings else None
        out = (N.TpchQ10Row * len(t["cmap"]))()
        n = C.c_int64()
        engine.ctx.call("bo_tpch_q10", C.byref(tb), start, end_, 2, 2, out, len(t["cmap"]), C.byref(n))
        want = q10_oracle(t, start, end_, 2, 2, 25)
        assert n.value == len(want[0])
        got = np.frombuffer(out, dtype=row_t)[: n.value]
        for name, w in zip(("rev", "cust", "crow", "nk"), want):
            assert np.array_equal(got[name], w), (name, start, end_)
        crow = want[2]
        assert np.array_equal(got["acct"], acct[crow] if strings else np.zeros_like(crow))
        for k in range(4):
            b = offs[k][crow] if strings else np.zeros_like(crow)
            ln = offs[k][crow + 1] - offs[k][crow] if strings else np.zeros_like(crow)
            assert np.array_equal(got[f"b{k}"], b) and np.array_equal(got[f"l{k}"], ln), k
    out = (N.TpchQ10Row * 1)()
    n = C.c_int64(-1)
    engine.ctx.call("bo_tpch_q10", C.byref(tb), 0, 2405, -1, 2, out, 1, C.byref(n))  # no 'R' in the dictionary
    assert n.value == 0


HOST_ROW = np.dtype([("cust", "<i4"), ("acct", "<i4"), ("rev", "<i8")] +
                    [(f"{f}_{x}", "<u8") for f in ("name", "nation", "address", "phone", "comment")
                     for x in ("ptr", "len")])


@pytest.mark.parametrize("n_customer", [150_000, 700_000])
def test_q10_host_rows_match_the_device_rows(engine, torch_cuda, n_customer):
    """bo_tpch_q10_host_rows writes each row, strings resolved to host
    pointers, into mapped pinned memory: the same rows as bo_tpch_q10 with
    every string pointing at base + begin of its column and every nation name
    at the given table's entry.  With 700k customers the full window has more
    result rows than one cluster sort holds (the sort is redone after the
    count is read back).  Pageable memory for the rows is refused."""
    torch = torch_cuda
    t = tables(1_500_000, 4, False, n_customer)
    g = dev(torch, t)
    no = len(t["okey"])
    begin, end = ranges(engine, torch, g, no)
    nc = len(t["cnation"])
    rng = np.random.default_rng(6)
    offs = [np.concatenate([[0], np.cumsum(rng.integers(0, 90, size=nc))]).astype(np.uint32) for _ in range(4)]
    acct = rng.integers(-99_999, 999_999, size=nc).astype(np.int32)
    offs_d = [torch.from_numpy(o).cuda() for o in offs]
    acct_d = torch.from_numpy(acct).cuda()
    tb = N.TpchQ10Tables()
    tb.o_orderkey, tb.o_custkey, tb.o_orderdate = g["okey"].data_ptr(), g["ocust"].data_ptr(), g["odate"].data_ptr()
    tb.o_li_begin, tb.o_li_end, tb.n_orders = begin.data_ptr(), end.data_ptr(), no
    tb.l_orderkey, tb.l_returnflag_linestatus = g["lkey"].data_ptr(), g["lcode"].data_ptr()
    tb.l_discounted_price, tb.n_lineitem = g["ldp"].data_ptr(), len(t["lkey"])
    tb.lineitem_orderkey_sorted = 1
    tb.nation_bound = 25
    tb.custkey_to_row, tb.n_custkey_map = g["cmap"].data_ptr(), len(t["cmap"])
    tb.c_nationkey, tb.n_customer = g["cnation"].data_ptr(), nc
    tb.c_name_offsets, tb.c_address_offsets, tb.c_phone_offsets, tb.c_comment_offsets = [o.data_ptr() for o in offs_d]
    tb.c_acctbal = acct_d.data_ptr()
    data = [C.create_string_buffer(int(o[-1]) + 1) for o in offs]  # host bytes the offsets index
    names = [C.create_string_buffer(f"NATION_{k:02d}".encode()) for k in range(25)]
    ntab = (N.HostStr * 25)(*[N.HostStr(C.addressof(b), 9) for b in names])
    hs = N.TpchQ10HostStrings(*[C.addressof(b) for b in data], C.addressof(ntab), 25, 0)
    cap = len(t["cmap"])
    assert C.sizeof(N.TpchQ10HostRow) == HOST_ROW.itemsize == 96
    mapped = C.c_void_p()
    engine.ctx.call("bo_host_alloc_pinned", HOST_ROW.itemsize * cap, C.byref(mapped))
    ref_t = np.dtype([("rev", "<i8"), ("cust", "<i4"), ("crow", "<i4"), ("nk", "<i4"), ("acct", "<i4"),
                      ("b0", "<u4"), ("l0", "<u4"), ("b1", "<u4"), ("l1", "<u4"), ("b2", "<u4"), ("l2", "<u4"),
                      ("b3", "<u4"), ("l3", "<u4")])
    bases = np.array([C.addressof(b) for b in data], np.uint64)
    nation_ptr = np.array([C.addressof(b) for b in names], np.uint64)
    sizes = []
    try:
        for start, end_ in [(640, 730), (0, 2405), (100, 100)]:
            ref = (N.TpchQ10Row * cap)()
            n_ref, n = C.c_int64(), C.c_int64(-1)
            engine.ctx.call("bo_tpch_q10", C.byref(tb), start, end_, 2, 2, ref, cap, C.byref(n_ref))
            engine.ctx.call("bo_tpch_q10_host_rows", C.byref(tb), start, end_, 2, 2, C.byref(hs), mapped, cap,
                            C.byref(n))
            assert n.value == n_ref.value
            sizes.append(n.value)
            a = np.frombuffer((C.c_char * (HOST_ROW.itemsize * cap)).from_address(mapped.value),
                              dtype=HOST_ROW)[: n.value]
            b = np.frombuffer(ref, dtype=ref_t)[: n.value]
            assert np.array_equal(a["cust"], b["cust"]) and np.array_equal(a["rev"], b["rev"])
            assert np.array_equal(a["acct"], b["acct"])
            for k, f in enumerate(("name", "address", "phone", "comment")):
                assert np.array_equal(a[f"{f}_ptr"], bases[k] + b[f"b{k}"].astype(np.uint64)), f
                assert np.array_equal(a[f"{f}_len"], b[f"l{k}"].astype(np.uint64)), f
            assert np.array_equal(a["nation_ptr"], nation_ptr[b["nk"]]) and (a["nation_len"] == 9).all()
        if n_customer > 150_000:
            assert max(sizes) > 131_072  # the pass-sequence rerun ran
        pageable = (N.TpchQ10HostRow * 4)()
        with pytest.raises(N.BoError) as e:
            engine.ctx.call("bo_tpch_q10_host_rows", C.byref(tb), 0, 2405, 2, 2, C.byref(hs), pageable, 4,
                            C.byref(n))
        assert e.value.status == -1
    finally:
        engine.ctx.call("bo_host_free_pinned", mapped)


def test_q18_error_contract(engine, torch_cuda):
    torch = torch_cuda
    okey = torch.arange(1, 1001, dtype=torch.int32, device="cuda")
    zeros16 = torch.zeros(1000, dtype=torch.int16, device="cuda")
    ones32 = torch.ones(1000, dtype=torch.int32, device="cuda")
    lkey = torch.arange(0, 1000, dtype=torch.int32, device="cuda")
    lkey[500] = 1001  # beyond the dense sum array
    qty = torch.full((1000,), 100, dtype=torch.int16, device="cuda")
    tb = N.TpchQ18Tables()
    tb.o_orderkey, tb.o_custkey, tb.o_orderdate, tb.o_totalprice = (okey.data_ptr(), ones32.data_ptr(),
                                                                     zeros16.data_ptr(), ones32.data_ptr())
    tb.n_orders, tb.l_orderkey, tb.l_quantity, tb.n_lineitem = 1000, lkey.data_ptr(), qty.data_ptr(), 1000
    tb.n_customer, tb.dense_orderkeys, tb.dense_custkeys = 1, 1, 1
    out = (N.TpchQ18Row * 1000)()
    n = C.c_int64()
    with pytest.raises(N.BoError) as e:
        engine.ctx.call("bo_tpch_q18", C.byref(tb), 50, out, 1000, C.byref(n))
    assert e.value.status == -6
    lkey[500] = 500
    engine.ctx.call("bo_tpch_q18", C.byref(tb), 50, out, 1000, C.byref(n))  # the context stays usable
    assert n.value == 999  # orderkeys 1..999 have one lineitem each; every order maps to customer row 0
    tb.l_orderkey = lkey.data_ptr() + 4
    tb.n_lineitem = 999
    with pytest.raises(N.BoError) as e:
        engine.ctx.call("bo_tpch_q18", C.byref(tb), 50, out, 1000, C.byref(n))
    assert e.value.status == -1


def q13_match(s: bytes, w1: bytes, w2: bytes) -> bool:
    """matches_pattern of bespoke_tpch/query_q13.cpp:68-83 (first word1, then word2 after it)."""
    n = len(s)
    p1 = s.find(w1) if w1 else 0
    if p1 < 0 or p1 == n:
        return False
    start = p1 + len(w1)
    p2 = s.find(w2, start) if w2 else start
    return p2 >= 0 and p2 != n


@pytest.mark.parametrize("words", [(b"ab", b"ba"), (b"", b""), (b"a", b""), (b"", b"\x00\xff"), (b"abcab", b"c")])
def test_q13_matches_python(engine, torch_cuda, words):
    torch = torch_cuda
    rng = np.random.default_rng(11)
    n_orders, n_customer = 300_000, 20_000
    lens = rng.integers(0, 40, n_orders)
    lens[rng.integers(0, n_orders, 200)] = rng.integers(3000, 9000, 200)  # warps whose comments overflow the slice
    alphabet = np.frombuffer(b"abc \x00\xff", np.uint8)
    data = alphabet[rng.integers(0, len(alphabet), int(lens.sum()))]
    offs = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint32)
    ocust = rng.integers(0, n_customer + 1, n_orders).astype(np.int32)
    ckey = rng.permutation(np.arange(1, n_customer + 1, dtype=np.int32))
    ckey[-3:] = ckey[:3]  # repeated customer rows count twice
    w1, w2 = words
    raw = data.tobytes()
    counts = np.zeros(n_customer + 1, np.int64)
    for i in range(n_orders):
        if not q13_match(raw[offs[i]:offs[i + 1]], w1, w2):
            counts[ocust[i]] += 1
    dist = np.bincount(counts[ckey])
    want = sorted(((c, d) for c, d in enumerate(dist) if d), key=lambda r: (-r[1], -r[0]))
    g = dev(torch, dict(data=data if len(data) else np.zeros(16, np.uint8), offs=offs.view(np.int32), ocust=ocust,
                        ckey=ckey))
    tb = N.TpchQ13Tables()
    tb.o_comment, tb.o_comment_offsets, tb.o_custkey = g["data"].data_ptr(), g["offs"].data_ptr(), g["ocust"].data_ptr()
    tb.n_orders, tb.c_custkey, tb.n_customer, tb.n_count_map = n_orders, g["ckey"].data_ptr(), n_customer, n_customer + 1
    out = (N.TpchQ13Row * (n_orders + 1))()
    n = C.c_int64()
    for _ in range(2):  # the histogram is left clear for the next call
        engine.ctx.call("bo_tpch_q13", C.byref(tb), w1, len(w1), w2, len(w2), out, n_orders + 1, C.byref(n))
        assert [(out[i].c_count, out[i].custdist) for i in range(n.value)] == want
