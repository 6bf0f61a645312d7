"""Q22 through the C ABI at 1.5M customers against a numpy restatement of
run_q22 (bespoke_tpch/query_q22.cpp:272-540): phone classes (numeric
prefixes, non-numeric two-byte prefixes, short phones), the integer average
of the allowed positive balances, customers above it without orders per
class; custkeys beyond the order custkeys' range (counted as without
orders).  Byte-level parity with the reference is in test_dropin_gpu.py."""
import ctypes as C

import numpy as np
import pytest

from bespokeolap_artifacts_b200 import native as N

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def q22_data(torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(22)
    n = 1_500_000
    key = rng.permutation(np.arange(1, n + 1, dtype=np.int32))
    bal = rng.integers(-99_999, 999_999, n).astype(np.int32)
    prefix = rng.integers(0, 100, n).astype(np.uint8)
    prefix[rng.random(n) < 0.05] = 255
    pair = (0x10000 | (rng.integers(65, 70, n) << 8) | rng.integers(65, 70, n)).astype(np.uint32)
    pair[rng.random(n) < 0.01] = 0  # phones shorter than two bytes
    n_order_keys = n - 1000  # the largest custkeys lie beyond the order custkeys
    has = rng.random(n_order_keys) < 0.6
    bits = np.packbits(has, bitorder="little")
    words = np.zeros((n_order_keys + 31) // 32 * 4, np.uint8)
    words[: len(bits)] = bits
    d = dict(key=key, bal=bal, prefix=prefix, pair=pair, words=words.view(np.uint32), has=has)
    g = {k: torch.from_numpy(v.view(np.int32) if v.dtype == np.uint32 else v).cuda()
         for k, v in d.items() if k != "has"}
    return d, g, n_order_keys


def restate(d, numeric, extra):
    cls = np.full(len(d["key"]), -1, np.int64)
    prefix = d["prefix"].astype(np.int64)
    num = prefix != 255
    cls[num] = np.where(numeric[np.minimum(prefix[num], 99)] == 1, prefix[num], -1)
    for i, e in enumerate(extra):
        m = (~num) & ((d["pair"] & 0x10000) != 0) & ((d["pair"] & 0xFFFF) == e)
        cls[m] = 100 + i
    ok = (cls >= 0) & (d["bal"] > 0)
    counts, sums = [0] * 107, [0] * 107
    if ok.sum() == 0:
        return counts, sums
    avg = int(d["bal"][ok].astype(np.int64).sum()) // int(ok.sum())
    k = d["key"].astype(np.int64)
    has = np.zeros(len(k), bool)
    inr = k < len(d["has"])
    has[inr] = d["has"][k[inr]]
    keep = ok & (d["bal"] > avg) & ~has
    for c in np.unique(cls[keep]):
        m = keep & (cls == c)
        counts[c], sums[c] = int(m.sum()), int(d["bal"][m].astype(np.int64).sum())
    return counts, sums


@pytest.mark.parametrize("codes", [([13, 31, 23], []), (list(range(100)), [0x4142, 0x4545]), ([], [0x4646]), ([7], [])])
def test_q22_matches_numpy(engine, q22_data, codes):
    d, g, n_order_keys = q22_data
    numeric = np.zeros(100, np.uint8)
    numeric[codes[0]] = 1
    extra = np.array(codes[1], np.uint16)
    t = N.TpchQ22Tables()
    t.c_custkey, t.c_acctbal = g["key"].data_ptr(), g["bal"].data_ptr()
    t.c_phone_prefix, t.c_phone_pair, t.n_customer = g["prefix"].data_ptr(), g["pair"].data_ptr(), len(d["key"])
    t.o_has_order, t.n_order_custkeys = g["words"].data_ptr(), n_order_keys
    counts, sums = (C.c_int64 * 107)(), (C.c_int64 * 107)()
    ex = extra.ctypes.data_as(C.c_void_p) if len(extra) else None
    engine.ctx.call("bo_tpch_q22", C.byref(t), numeric.tobytes(), ex, len(extra), counts, sums)
    want_c, want_s = restate(d, numeric, list(extra))
    assert list(counts) == want_c and list(sums) == want_s


def test_q22_arguments(engine):
    t = N.TpchQ22Tables()
    counts, sums = (C.c_int64 * 107)(), (C.c_int64 * 107)()
    extra = np.zeros(8, np.uint16)
    with pytest.raises(N.BoError):
        engine.ctx.call("bo_tpch_q22", C.byref(t), bytes(100), extra.ctypes.data_as(C.c_void_p), 8, counts, sums)
    t.n_customer = 4
    with pytest.raises(N.BoError):
        engine.ctx.call("bo_tpch_q22", C.byref(t), bytes(100), None, 0, counts, sums)  # null columns
