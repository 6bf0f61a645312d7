"""Q12 through the C ABI at 6M lineitems against a numpy restatement of
run_q12 (bespoke_tpch/query_q12.cpp:162-360), with and without the
per-lineitem shard maxima that carry the reference's shard pruning
(:265-270); plus the entry point's argument contract.  Byte-level parity with
the reference itself is in test_dropin_gpu.py."""
import ctypes as C

import numpy as np
import pytest

from bespokeolap_artifacts_b200 import native as N

pytestmark = pytest.mark.gpu


def data(n_orders: int, seed: int):
    rng = np.random.default_rng(seed)
    okey = (np.arange(n_orders, dtype=np.int64) // 8 * 32 + np.arange(n_orders) % 8 + 1).astype(np.int32)
    odate = np.sort(rng.integers(0, 2405, n_orders)).astype(np.int16)
    prio = rng.integers(0, 5, n_orders).astype(np.uint16)
    omap = np.full(int(okey.max()) + 1, -1, np.int32)
    omap[okey] = np.arange(n_orders, dtype=np.int32)
    lines = rng.integers(1, 8, n_orders)
    lkey = np.repeat(okey, lines)
    ld = np.repeat(odate, lines).astype(np.int32)
    n = len(lkey)
    lkey[rng.integers(0, n, 500)] = rng.integers(1, 1 << 30, 500)  # orderkeys without an order
    ship = ld + rng.integers(1, 122, n)
    commit = ld + rng.integers(30, 91, n)
    receipt = ship + rng.integers(1, 61, n)  # some received more than 30 days after shipping
    mode = rng.integers(0, 7, n).astype(np.uint16)
    cr = ((receipt.astype(np.uint32) & 0xFFFF) << 16) | (commit.astype(np.uint32) & 0xFFFF)
    shard = rng.integers(0, 400, n)  # arbitrary shard ids; their latest shipdates
    smax = np.full(400, -32768, np.int64)
    np.maximum.at(smax, shard, ship)
    return dict(mode=mode, cr=cr.astype(np.uint32), ship=ship.astype(np.int16), lkey=lkey,
                smax=smax[shard].astype(np.int16), omap=omap, prio=prio)


def restate(d, c1, c2, h1, h2, start, end, use_shards):
    commit = (d["cr"] & 0xFFFF).astype(np.uint16).view(np.int16).astype(np.int32)
    receipt = (d["cr"] >> 16).astype(np.uint16).view(np.int16).astype(np.int32)
    ship = d["ship"].astype(np.int32)
    m = d["mode"].astype(np.int32)
    ok = ((m == c1) | (m == c2)) & (commit < receipt) & (ship < commit)
    ok &= (receipt - start).astype(np.uint32) < np.uint32(end - start)
    if use_shards:
        ok &= d["smax"].astype(np.int32) >= start - 30
    key = d["lkey"].astype(np.int64)
    inmap = (key >= 0) & (key < len(d["omap"]))
    row = np.where(inmap, d["omap"][np.where(inmap, key, 0)], -1)
    ok &= row >= 0
    pc = d["prio"][np.where(ok, row, 0)].astype(np.int32)
    high = (pc == h1) | (pc == h2)
    out = []
    for c in (c1, c2):
        sel = ok & (m == c)
        out += [int((sel & high).sum()), int((sel & ~high).sum())]
    return out


@pytest.fixture(scope="module")
def q12_device(torch_cuda):
    torch = torch_cuda
    d = data(1_500_000, 3)
    g = {k: torch.from_numpy(v.view(np.int16) if v.dtype == np.uint16 else
                             (v.view(np.int32) if v.dtype == np.uint32 else v)).cuda() for k, v in d.items()}
    return d, g


@pytest.mark.parametrize("use_shards", [False, True])
@pytest.mark.parametrize("codes", [(0, 3, 0, 1), (5, -1, 2, -1), (-1, 6, 4, 0), (2, 4, -1, -1)])
@pytest.mark.parametrize("window", [(730, 1095), (0, 366), (2300, 2665)])
def test_q12_matches_numpy(engine, q12_device, use_shards, codes, window):
    d, g = q12_device
    c1, c2, h1, h2 = codes
    start, end = window
    t = N.TpchQ12Tables()
    t.l_shipmode, t.l_commit_receipt, t.l_shipdate = g["mode"].data_ptr(), g["cr"].data_ptr(), g["ship"].data_ptr()
    t.l_orderkey = g["lkey"].data_ptr()
    t.l_shard_max_shipdate = g["smax"].data_ptr() if use_shards else None
    t.n_lineitem = len(d["mode"])
    t.orderkey_to_row, t.n_orderkey_map = g["omap"].data_ptr(), len(d["omap"])
    t.o_orderpriority, t.n_orders = g["prio"].data_ptr(), len(d["prio"])
    counts = (C.c_int64 * 4)()
    engine.ctx.call("bo_tpch_q12", C.byref(t), c1, c2, h1, h2, start, end, counts)
    assert list(counts) == restate(d, c1, c2, h1, h2, start, end, use_shards)


def test_q12_arguments(engine, q12_device):
    d, g = q12_device
    t = N.TpchQ12Tables()
    t.n_lineitem = 8
    counts = (C.c_int64 * 4)()
    with pytest.raises(N.BoError):
        engine.ctx.call("bo_tpch_q12", C.byref(t), 0, 1, 0, 1, 0, 10, counts)  # null columns
    t.l_shipmode, t.l_commit_receipt = g["mode"].data_ptr() + 2, g["cr"].data_ptr()
    t.l_shipdate, t.l_orderkey = g["ship"].data_ptr(), g["lkey"].data_ptr()
    with pytest.raises(N.BoError):
        engine.ctx.call("bo_tpch_q12", C.byref(t), 0, 1, 0, 1, 0, 10, counts)  # misaligned shipmode codes
    t.l_shipmode, t.n_lineitem = g["mode"].data_ptr(), 0
    engine.ctx.call("bo_tpch_q12", C.byref(t), 0, 1, 0, 1, 0, 10, counts)
    assert list(counts) == [0, 0, 0, 0]
