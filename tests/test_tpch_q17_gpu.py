"""Q17 through the C ABI at 6M lineitems / 200k parts against a numpy
restatement of run_q17 (bespoke_tpch/query_q17.cpp:119-311): the parts of
one brand and container, their lineitems' quantity sums and counts, and the
extended prices of lineitems below a fifth of their part's average; part
rows with keys outside [0, max], duplicate part keys, lineitem partkeys
beyond the largest part key and negative ones (no part).  Byte-level parity
of the formatted result with the reference is in test_dropin_gpu.py."""
import ctypes as C

import numpy as np
import pytest

from bespokeolap_artifacts_b200 import native as N

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def q17_data(torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(17)
    n_part, n = 200_000, 6_000_005
    pkey = rng.permutation(np.arange(1, n_part + 1, dtype=np.int32))
    pkey[:50] = rng.integers(-3, 0, 50)  # rows with keys no lineitem bit covers
    brand = rng.integers(0, 25, n_part).astype(np.uint16)
    cont = rng.integers(0, 40, n_part).astype(np.uint16)
    lpk = rng.integers(-2, n_part + 300, n).astype(np.int32)
    qty = (rng.integers(1, 51, n) * 100).astype(np.int16)
    price = rng.integers(90_000, 10_500_000, n).astype(np.int32)
    d = dict(pkey=pkey, brand=brand, cont=cont, lpk=lpk, qty=qty, price=price)
    g = {k: torch.from_numpy(v.view(np.int16) if v.dtype == np.uint16 else v).cuda() for k, v in d.items()}
    return d, g


def restate(d, b, c):
    max_key = int(d["pkey"].max())
    match = np.zeros(max_key + 1, bool)
    sel = (d["pkey"] >= 0) & (d["brand"] == b) & (d["cont"] == c)
    match[d["pkey"][sel]] = True
    k = d["lpk"].astype(np.int64)
    hit = (k >= 0) & (k <= max_key)
    hit[hit] = match[k[hit]]
    qty = d["qty"].astype(np.int64)
    s = np.bincount(k[hit], weights=qty[hit], minlength=max_key + 1).astype(np.int64)
    cnt = np.bincount(k[hit], minlength=max_key + 1).astype(np.int64)
    keep = hit.copy()
    keep[hit] = qty[hit] * 5 * cnt[k[hit]] < s[k[hit]]
    return int(d["price"][keep].astype(np.int64).sum())


@pytest.mark.parametrize("codes", [(3, 7), (0, 0), (24, 39), (30, 1)])
def test_q17_matches_numpy(engine, q17_data, codes):
    d, g = q17_data
    t = N.TpchQ17Tables()
    t.l_partkey, t.l_quantity, t.l_extendedprice = g["lpk"].data_ptr(), g["qty"].data_ptr(), g["price"].data_ptr()
    t.n_lineitem = len(d["lpk"])
    t.p_partkey, t.p_brand, t.p_container = g["pkey"].data_ptr(), g["brand"].data_ptr(), g["cont"].data_ptr()
    t.n_part, t.max_partkey = len(d["pkey"]), int(d["pkey"].max())
    out = C.c_int64()
    for _ in range(2):  # workspace reused
        engine.ctx.call("bo_tpch_q17", C.byref(t), codes[0], codes[1], C.byref(out))
        assert out.value == restate(d, *codes)


def test_q17_arguments(engine, q17_data):
    d, g = q17_data
    t = N.TpchQ17Tables()
    t.n_lineitem, t.n_part, t.max_partkey = 8, 1, 5
    out = C.c_int64()
    with pytest.raises(N.BoError):
        engine.ctx.call("bo_tpch_q17", C.byref(t), 0, 0, C.byref(out))  # null columns
    t.l_partkey, t.l_quantity, t.l_extendedprice = g["lpk"].data_ptr() + 4, g["qty"].data_ptr(), g["price"].data_ptr()
    t.p_partkey, t.p_brand, t.p_container = g["pkey"].data_ptr(), g["brand"].data_ptr(), g["cont"].data_ptr()
    with pytest.raises(N.BoError):
        engine.ctx.call("bo_tpch_q17", C.byref(t), 0, 0, C.byref(out))  # misaligned partkeys
