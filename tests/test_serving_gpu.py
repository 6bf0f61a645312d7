"""Serving with continuous batching: every request's answer is the same as
its answer alone (exact), for batches formed from a Poisson stream, with
under-predicted tables (exact reruns) and with the one-pipeline-per-launch
baseline."""
import numpy as np
import pytest

from bespokeolap_artifacts_b200 import batching as B
from bespokeolap_artifacts_b200 import serving as S

pytestmark = pytest.mark.gpu


class LowSizer:
    """Stand-in sizer predicting one row / group: every presized table is far
    too small, so every join and group-by instance overflows and is rerun."""

    def predict_host(self, x):
        return np.ones((len(x), 2))[:, 0] if x.shape[1] == 8 else np.ones((len(x), 2))


@pytest.fixture(scope="module")
def tables(engine, torch_cuda):
    return S.ServingTables.load(engine, fact_rows=400_000, seed=3)


def check(engine, tables, reqs):
    for r in reqs:
        solo = B.solo_result(engine, S.instance_of(tables, r))
        assert B.same_answer(r.result, solo), (r.rid, r.kind, r.params)


def test_served_results_equal_solo(engine, tables):
    reqs = S.poisson_requests(20000.0, 48, seed=7)
    srv = S.BatchedServer(tables, n_slots=2, max_batch=8, pool_bytes=512 << 20, max_items=32768)
    srv.serve(reqs)
    assert srv.launches < len(reqs)  # requests shared launches
    check(engine, tables, reqs)
    st = S.latency_stats(reqs)
    assert st["p99_ms"] >= st["p50_ms"] > 0
    srv.close()


def test_served_with_overflowing_predictions(engine, tables):
    reqs = S.poisson_requests(20000.0, 24, seed=8, mix=(0, 1, 1))
    srv = S.BatchedServer(tables, n_slots=2, max_batch=6, pool_bytes=512 << 20, max_items=32768,
                          join_sizer=LowSizer(), gb_sizer=LowSizer())
    srv.serve(reqs)
    assert any(r.result.get("reruns", 0) for r in reqs)
    check(engine, tables, reqs)
    srv.close()


def test_one_per_launch_baseline(engine, tables):
    reqs = S.poisson_requests(5000.0, 12, seed=9)
    S.serve_one_per_launch(engine, tables, reqs)
    check(engine, tables, reqs)


def test_served_joins_share_one_pass(engine, tables):
    reqs = S.poisson_requests(50000.0, 40, seed=10, mix=(0, 1, 0))
    srv = S.BatchedServer(tables, n_slots=2, max_batch=16, pool_bytes=512 << 20, max_items=32768)
    srv.serve(reqs)
    assert srv.launches < len(reqs)
    assert all(r.result.get("reruns", 0) == 0 for r in reqs)
    check(engine, tables, reqs)
    srv.close()


def test_served_without_sharing(engine, tables):
    reqs = S.poisson_requests(20000.0, 24, seed=11)
    srv = S.BatchedServer(tables, n_slots=2, max_batch=8, pool_bytes=512 << 20, max_items=32768, shared=False)
    srv.serve(reqs)
    check(engine, tables, reqs)
    srv.close()


@pytest.mark.parametrize("policy,slots,spill,batch_from", [("short_first", 2, 1, 1), ("short_first", 3, 1, 1),
                                                           ("short_first", 2, 3, 1), ("fifo", 2, 2, 1),
                                                           ("short_first", 2, 1, 3), ("fifo", 1, 1, 4)])
def test_served_short_first_equals_solo(engine, tables, policy, slots, spill, batch_from):
    """Short-first admission (one kind per launch, shortest kind first, no
    starvation), the spill rule (a second slot starts only once requests
    queue) and the batch threshold (one request per launch while fewer than
    batch_from wait): answers unchanged, every request served."""
    reqs = S.poisson_requests(20000.0, 60, seed=12)
    srv = S.BatchedServer(tables, n_slots=slots, max_batch=8, pool_bytes=512 << 20, max_items=32768,
                          policy=policy, max_wait_ms=1.0, spill_queue=spill, batch_from=batch_from)
    srv.serve(reqs)
    assert all(r.result is not None and r.done >= r.arrival for r in reqs)
    check(engine, tables, reqs)
    srv.close()


def test_served_lone_requests_at_low_rate(engine, tables):
    """At a low arrival rate every request finds an idle slot: scan-agg runs
    alone through its kernel and each join in two phases (exact count, then
    the join sized from it, the serve loop never waiting on the device)."""
    reqs = S.poisson_requests(300.0, 18, seed=13, mix=(1, 2, 0))
    srv = S.BatchedServer(tables, n_slots=2, max_batch=8, pool_bytes=512 << 20, max_items=32768)
    srv.serve(reqs)
    assert srv.launches == len(reqs)
    assert all(r.result.get("reruns", 0) == 0 for r in reqs)
    check(engine, tables, reqs)
    srv.close()
