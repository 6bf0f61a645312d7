"""Q11 through the C ABI at 800k partsupp rows against a numpy restatement of
run_q11's sums (bespoke_tpch/query_q11.cpp:109-224): per-partkey and total
stock value of the nation's suppliers, partkeys from a negative minimum,
suppkeys outside the supplier table.  Byte-level parity of the formatted
result with the reference is in test_dropin_gpu.py."""
import ctypes as C

import numpy as np
import pytest

from bespokeolap_artifacts_b200 import native as N

pytestmark = pytest.mark.gpu


def test_q11_matches_numpy(engine, torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(11)
    n = 800_003
    pk = np.sort(rng.integers(-50, 200_000, n)).astype(np.int32)
    sk = rng.integers(-2, 10_050, n).astype(np.int32)
    val = rng.integers(100, 999_900_000, n).astype(np.int32)
    in_nation = (rng.random(10_000) < 0.04).astype(np.uint8)
    g = {k: torch.from_numpy(v).cuda() for k, v in dict(pk=pk, sk=sk, val=val).items()}
    t = N.TpchQ11Tables()
    t.ps_partkey, t.ps_suppkey, t.ps_value, t.n_partsupp = g["pk"].data_ptr(), g["sk"].data_ptr(), g["val"].data_ptr(), n
    t.min_partkey, t.max_partkey = int(pk[0]), int(pk[-1])
    rng_n = int(pk[-1]) - int(pk[0]) + 1
    sums = (C.c_int64 * rng_n)()
    total = C.c_int64()
    engine.ctx.call("bo_tpch_q11", C.byref(t), in_nation.tobytes(), len(in_nation), sums, C.byref(total))
    k = sk.astype(np.int64)
    ok = (k >= 0) & (k < len(in_nation))
    ok[ok] = in_nation[k[ok]].astype(bool)
    want = np.zeros(rng_n, np.int64)
    np.add.at(want, (pk[ok].astype(np.int64) - int(pk[0])), val[ok].astype(np.int64))
    assert total.value == int(val[ok].astype(np.int64).sum())
    assert np.array_equal(np.ctypeslib.as_array(sums), want)


def test_q11_arguments(engine):
    t = N.TpchQ11Tables()
    t.n_partsupp, t.min_partkey, t.max_partkey = 4, 5, 1
    total = C.c_int64()
    sums = (C.c_int64 * 4)()
    with pytest.raises(N.BoError):
        engine.ctx.call("bo_tpch_q11", C.byref(t), bytes(4), 4, sums, C.byref(total))  # empty key range


@pytest.mark.parametrize("rate,fraction", [(0.04, 0.00001), (0.5, 0.0)])
@pytest.mark.parametrize("mapped", [False, True])
def test_q11_rows_match_numpy(engine, torch_cuda, rate, fraction, mapped):
    """bo_tpch_q11_rows: the non-zero part sums above (double)total * fraction,
    by value descending then partkey (query_q11.cpp:186-210).  With half the
    suppliers in the nation and fraction 0 about 188k parts qualify, more
    than one cluster sort holds (the sort is redone after the count is read
    back); rows into pageable and into mapped pinned memory."""
    torch = torch_cuda
    rng = np.random.default_rng(12)
    n = 800_003
    pk = np.sort(rng.integers(-50, 200_000, n)).astype(np.int32)
    sk = rng.integers(-2, 10_050, n).astype(np.int32)
    val = rng.integers(100, 999_900_000, n).astype(np.int32)
    in_nation = (rng.random(10_000) < rate).astype(np.uint8)
    g = {k: torch.from_numpy(v).cuda() for k, v in dict(pk=pk, sk=sk, val=val).items()}
    t = N.TpchQ11Tables()
    t.ps_partkey, t.ps_suppkey, t.ps_value, t.n_partsupp = g["pk"].data_ptr(), g["sk"].data_ptr(), g["val"].data_ptr(), n
    t.min_partkey, t.max_partkey = int(pk[0]), int(pk[-1])
    rng_n = int(pk[-1]) - int(pk[0]) + 1
    k = sk.astype(np.int64)
    ok = (k >= 0) & (k < len(in_nation))
    ok[ok] = in_nation[k[ok]].astype(bool)
    sums = np.zeros(rng_n, np.int64)
    np.add.at(sums, (pk[ok].astype(np.int64) - int(pk[0])), val[ok].astype(np.int64))
    total = int(val[ok].astype(np.int64).sum())
    keep = np.nonzero((sums != 0) & (sums.astype(np.float64) > float(total) * fraction))[0]
    order = np.lexsort((keep, -sums[keep]))
    want_pk, want_v = keep[order] + int(pk[0]), sums[keep[order]]
    row_t = np.dtype([("pk", "<i4"), ("pad", "<i4"), ("v", "<i8")])
    nr = C.c_int64(-1)
    if mapped:
        buf = C.c_void_p()
        engine.ctx.call("bo_host_alloc_pinned", row_t.itemsize * rng_n, C.byref(buf))
        try:
            engine.ctx.call("bo_tpch_q11_rows", C.byref(t), in_nation.tobytes(), len(in_nation), fraction,
                            C.cast(buf, C.POINTER(N.TpchQ11Row)), rng_n, C.byref(nr))
            got = np.frombuffer((C.c_char * (row_t.itemsize * rng_n)).from_address(buf.value), dtype=row_t).copy()
        finally:
            engine.ctx.call("bo_host_free_pinned", buf)
    else:
        out = (N.TpchQ11Row * rng_n)()
        engine.ctx.call("bo_tpch_q11_rows", C.byref(t), in_nation.tobytes(), len(in_nation), fraction, out, rng_n,
                        C.byref(nr))
        got = np.frombuffer(out, dtype=row_t)
    assert nr.value == len(want_pk)
    if rate > 0.1:
        assert nr.value > 131_072
    got = got[: nr.value]
    assert np.array_equal(got["pk"], want_pk) and np.array_equal(got["v"], want_v)
