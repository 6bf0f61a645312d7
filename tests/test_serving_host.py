"""Host logic of the serving loop (no GPU): the Poisson request stream and
admission by footprint in arrival order."""
from collections import deque

import numpy as np

from bespokeolap_artifacts_b200 import native as N
from bespokeolap_artifacts_b200 import serving as S


def test_poisson_stream_is_seeded_and_ordered():
    a = S.poisson_requests(1000.0, 2000, seed=5)
    b = S.poisson_requests(1000.0, 2000, seed=5)
    assert [(r.kind, r.params, r.arrival) for r in a] == [(r.kind, r.params, r.arrival) for r in b]
    t = np.array([r.arrival for r in a])
    assert np.all(np.diff(t) > 0)
    assert abs(len(a) / t[-1] - 1000.0) < 100.0  # mean rate
    kinds = {r.kind for r in a}
    assert kinds == {N.BATCH_SCAN_AGG, N.BATCH_JOIN, N.BATCH_GROUPBY}
    assert S.poisson_requests(1000.0, 100, seed=5, mix=(0, 1, 0))[0].kind == N.BATCH_JOIN


def test_admission_by_footprint_in_arrival_order():
    reqs = [S.Request(i, N.BATCH_JOIN, {}, float(i)) for i in range(6)]
    foot = {0: (100, 10), 1: (300, 10), 2: (50, 10), 3: (10, 10), 4: (10, 10), 5: (10, 10)}
    q = deque(reqs)
    got = S.admit(q, foot, max_batch=8, pool_bytes=400, max_items=1000)
    assert [r.rid for r in got] == [0, 1]          # request 2 would exceed 400 bytes: it waits (FIFO)
    got = S.admit(q, foot, max_batch=2, pool_bytes=400, max_items=1000)
    assert [r.rid for r in got] == [2, 3]          # batch size limit
    got = S.admit(q, foot, max_batch=8, pool_bytes=400, max_items=15)
    assert [r.rid for r in got] == [4]             # work-item limit
    big = deque([S.Request(9, N.BATCH_JOIN, {}, 0.0)])
    got = S.admit(big, {9: (10_000, 5)}, max_batch=8, pool_bytes=400, max_items=1000)
    assert [r.rid for r in got] == [9]             # alone, never starved


def test_latency_stats():
    reqs = [S.Request(i, 0, {}, i * 0.001) for i in range(100)]
    for r in reqs:
        r.done = r.arrival + 0.002
    st = S.latency_stats(reqs)
    assert abs(st["p50_ms"] - 2.0) < 1e-9 and abs(st["p99_ms"] - 2.0) < 1e-9 and st["requests"] == 100


def test_admission_of_one_kind_keeps_the_others_in_order():
    kinds = [N.BATCH_GROUPBY, N.BATCH_SCAN_AGG, N.BATCH_JOIN, N.BATCH_SCAN_AGG, N.BATCH_GROUPBY]
    q = deque(S.Request(i, k, {}, float(i)) for i, k in enumerate(kinds))
    foot = {i: (10, 10) for i in range(5)}
    got = S.admit(q, foot, max_batch=8, pool_bytes=400, max_items=1000, kind=N.BATCH_SCAN_AGG)
    assert [r.rid for r in got] == [1, 3]
    assert [r.rid for r in q] == [0, 2, 4]          # the rest keep arrival order
    got = S.admit(q, foot, max_batch=1, pool_bytes=400, max_items=1000, kind=N.BATCH_GROUPBY)
    assert [r.rid for r in got] == [0] and [r.rid for r in q] == [2, 4]


def test_short_first_picks_the_shortest_kind_unless_the_oldest_waited_too_long():
    q = deque([S.Request(0, N.BATCH_GROUPBY, {}, 0.0), S.Request(1, N.BATCH_JOIN, {}, 0.1),
               S.Request(2, N.BATCH_SCAN_AGG, {}, 0.2)])
    assert S.next_kind(q, "fifo", 0.0, 4.0) is None
    assert S.next_kind(q, "short_first", 1.0, 4.0) == N.BATCH_SCAN_AGG
    assert S.next_kind(q, "short_first", 5.0, 4.0) == N.BATCH_GROUPBY   # no starvation
    q.pop()
    assert S.next_kind(q, "short_first", 1.0, 4.0) == N.BATCH_JOIN
    assert S.next_kind(deque(), "short_first", 1.0, 4.0) is None
