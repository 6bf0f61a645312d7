"""The streamed join over pinned host columns (dense columns copied in
chunks, sparse columns read in place) returns the same answer as the
device-resident exact form and the oracle, in both sizing forms, for empty
and ragged inputs and an undersized prediction (exact rerun)."""
import numpy as np
import pytest

from bespokeolap_artifacts_b200 import datagen as dg
from bespokeolap_artifacts_b200.engine import PinnedColumns, join_stream
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FIELDS = ("build_rows", "distinct_keys", "match_count", "sum_exact", "sum_trunc")


def pinned(engine, j):
    return PinnedColumns(engine, {"b_key": j.b_key, "b_date": j.b_date, "b_seg": j.b_seg, "p_fk": j.p_fk,
                                  "p_price": j.p_price, "p_disc": j.p_disc})


@pytest.mark.parametrize("nb,np_", [(0, 0), (1000, 0), (0, 5000), (1, 1), (12345, 3_000_001), (1_500_000, 6_000_000)])
def test_stream_matches_oracle(engine, torch_cuda, nb, np_):
    torch = torch_cuda
    j = dg.gen_join(nb, np_, seed=nb + np_)
    pc = pinned(engine, j)
    try:
        ref = O.join_agg(j)
        plain = join_stream(engine, pc, nb, np_, j.date_lt, j.seg_eq)
        pred = torch.tensor([float(ref["build_count"])], dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        presized = join_stream(engine, pc, nb, np_, j.date_lt, j.seg_eq, pred)
        for r in (plain, presized):
            assert (r["build_rows"], r["match_count"], r["sum_exact"], r["sum_trunc"]) == \
                (ref["build_count"], ref["match_count"], ref["sum_exact"], ref["sum_trunc"])
        assert plain["mode"] == 0 and presized["mode"] == 1 and presized["reruns"] == 0
    finally:
        pc.close()


def test_stream_undersized_prediction_reruns(engine, torch_cuda):
    torch = torch_cuda
    j = dg.gen_join(400_000, 1_000_000, seed=7, date_lt=dg.DATE_HI)  # every date qualifies
    pc = pinned(engine, j)
    try:
        pred = torch.tensor([10.0], dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        r = join_stream(engine, pc, j.n_build, j.n_probe, j.date_lt, j.seg_eq, pred)
        ref = O.join_agg(j)
        assert r["reruns"] == 1 and r["match_count"] == ref["match_count"] and r["sum_exact"] == ref["sum_exact"]
    finally:
        pc.close()


def test_stream_rejects_pageable_host_memory(engine, torch_cuda):
    import ctypes as C

    from bespokeolap_artifacts_b200 import native as N

    j = dg.gen_join(1000, 1000, seed=1)
    b = N.JoinBuildCols(j.b_key.ctypes.data, j.b_date.ctypes.data, j.b_seg.ctypes.data, 1000)
    p = N.JoinProbeCols(j.p_fk.ctypes.data, j.p_price.ctypes.data, j.p_disc.ctypes.data, 1000)
    with pytest.raises(N.BoError):
        engine.ctx.call("bo_join_stream_host", C.byref(b), C.byref(p), C.byref(N.JoinParams(j.date_lt, j.seg_eq)),
                        None, C.byref(N.JoinResult()))


def test_stream_async_pipelined_queries(engine, torch_cuda):
    """Several queries in flight (two inputs alternating, two buffer sets):
    every result lands intact once the stream is synchronised."""
    import ctypes as C

    from bespokeolap_artifacts_b200 import native as N
    from bespokeolap_artifacts_b200.engine import join_stream_async

    torch = torch_cuda
    js = [dg.gen_join(200_000, 2_500_000, seed=21), dg.gen_join(300_000, 1_000_000, seed=22)]
    pcs = [pinned(engine, j) for j in js]
    refs = [O.join_agg(j) for j in js]
    sz = C.sizeof(N.JoinResult)
    out = C.c_void_p()
    engine.ctx.call("bo_host_alloc_pinned", C.c_size_t(8 * sz), C.byref(out))
    try:
        preds = torch.tensor([float(r["build_count"]) for r in refs], dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        for i in range(8):
            k = i % 2
            join_stream_async(engine, pcs[k], js[k].n_build, js[k].n_probe, js[k].date_lt, js[k].seg_eq,
                              preds[k:k + 1], out.value + i * sz)
        engine.ctx.call("bo_check_errors")
        for i in range(8):
            r = N.JoinResult.from_address(out.value + i * sz).as_dict()
            ref = refs[i % 2]
            assert (r["match_count"], r["sum_exact"], r["sum_trunc"], r["overflowed"]) == \
                (ref["match_count"], ref["sum_exact"], ref["sum_trunc"], 0), i
    finally:
        engine.ctx.call("bo_host_free_pinned", out)
        for pc in pcs:
            pc.close()


@pytest.mark.parametrize("threads", [0, 1, 3, -1])
def test_stream_host_gather_thread_counts(engine, torch_cuda, threads):
    """The payload of matching probe rows read in place (0 threads) or
    gathered on 1, 3 or the machine's default number of host threads: the same
    answer as the oracle, over several chunks (the last one ragged) and build
    keys that repeat (multiplicities above 1 travel with the match list)."""
    import dataclasses

    torch = torch_cuda
    j = dg.gen_join(300_000, 2 * (1 << 20) + 4321, seed=31)
    j = dataclasses.replace(j, b_key=(j.b_key % 200_000 + 1).astype(np.int32))  # each key about 1.5 times
    pc = pinned(engine, j)
    before = engine.host_threads
    try:
        engine.host_threads = threads
        assert engine.host_threads == threads or (threads < 0 and engine.host_threads >= 1)
        ref = O.join_agg(j)
        plain = join_stream(engine, pc, j.n_build, j.n_probe, j.date_lt, j.seg_eq)
        pred = torch.tensor([float(ref["build_count"])], dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        presized = join_stream(engine, pc, j.n_build, j.n_probe, j.date_lt, j.seg_eq, pred)
        qual = (j.b_seg == j.seg_eq) & (j.b_date < j.date_lt)
        distinct = int(np.unique(j.b_key[qual]).size)
        assert distinct < int(qual.sum())  # some qualifying keys do repeat
        for r in (plain, presized):
            assert (r["build_rows"], r["distinct_keys"], r["match_count"], r["sum_exact"], r["sum_trunc"]) == \
                (ref["build_count"], distinct, ref["match_count"], ref["sum_exact"], ref["sum_trunc"])
    finally:
        engine.host_threads = before
        pc.close()


def test_stream_host_gather_reports_bad_payload(engine, torch_cuda):
    """A matching probe row whose price lies outside the exact-arithmetic
    contract (>= 2^31) is reported by the gather's summing kernel as a data
    error when the queued work is drained; the context stays usable."""
    from bespokeolap_artifacts_b200 import native as N

    j = dg.gen_join(50_000, 400_000, seed=41, date_lt=dg.DATE_HI)
    ok = O.join_agg(j)
    bad = j.p_price.copy()
    matched = np.flatnonzero(np.isin(j.p_fk, j.b_key[(j.b_seg == j.seg_eq) & (j.b_date < j.date_lt)]))
    assert matched.size > 0
    bad[matched[matched.size // 2]] = 1 << 40
    pc_bad = PinnedColumns(engine, {"b_key": j.b_key, "b_date": j.b_date, "b_seg": j.b_seg, "p_fk": j.p_fk,
                                    "p_price": bad, "p_disc": j.p_disc})
    pc = pinned(engine, j)
    before = engine.host_threads
    try:
        engine.host_threads = 2
        with pytest.raises(N.BoError) as ei:
            join_stream(engine, pc_bad, j.n_build, j.n_probe, j.date_lt, j.seg_eq)
        assert ei.value.status == N.BO_ERR_DATA
        r = join_stream(engine, pc, j.n_build, j.n_probe, j.date_lt, j.seg_eq)
        assert (r["match_count"], r["sum_exact"]) == (ok["match_count"], ok["sum_exact"])
    finally:
        engine.host_threads = before
        pc_bad.close()
        pc.close()


def test_stream_async_thread_count_change_between_queries(engine, torch_cuda):
    """Queries queued on the host-gather form, a change of the thread count
    (which drains them), then queries read in place: every result intact."""
    import ctypes as C

    from bespokeolap_artifacts_b200 import native as N
    from bespokeolap_artifacts_b200.engine import join_stream_async

    torch = torch_cuda
    j = dg.gen_join(200_000, 1_500_000, seed=51)
    ref = O.join_agg(j)
    pc = pinned(engine, j)
    sz = C.sizeof(N.JoinResult)
    out = C.c_void_p()
    engine.ctx.call("bo_host_alloc_pinned", C.c_size_t(6 * sz), C.byref(out))
    before = engine.host_threads
    try:
        pred = torch.tensor([float(ref["build_count"])], dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        for i in range(6):
            if i == 3:
                engine.host_threads = 0
            join_stream_async(engine, pc, j.n_build, j.n_probe, j.date_lt, j.seg_eq, pred, out.value + i * sz)
        engine.ctx.call("bo_check_errors")
        for i in range(6):
            r = N.JoinResult.from_address(out.value + i * sz).as_dict()
            assert (r["match_count"], r["sum_exact"], r["sum_trunc"], r["overflowed"]) == \
                (ref["match_count"], ref["sum_exact"], ref["sum_trunc"], 0), i
    finally:
        engine.host_threads = before
        engine.ctx.call("bo_host_free_pinned", out)
        pc.close()
