"""The radix-partitioned filtered join (bo_join_partitioned*) gives the
oracle's answer exactly -- the restated filtered join of run_q3
(bespoke_tpch/query_q3.cpp:182-260) -- at every fan-out, with repeated build
keys (multiplicities), empty sides, and partitions whose tables are too small
(exact single-pass rerun)."""
import numpy as np
import pytest

from bespokeolap_artifacts_b200 import datagen as dg
from bespokeolap_artifacts_b200 import native as N
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FIELDS = ("build_rows", "distinct_keys", "match_count", "sum_exact", "sum_trunc")


def device(torch, j):
    b = [torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (j.b_key, j.b_date, j.b_seg)]
    p = [torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (j.p_fk, j.p_price, j.p_disc)]
    return b, p


def want(j):
    r = O.join_agg(j)
    distinct = len(np.unique(j.b_key[(j.b_date < j.date_lt) & (j.b_seg == j.seg_eq)]))
    return (r["build_count"], distinct, r["match_count"], r["sum_exact"], r["sum_trunc"])


# (build rows, probe rows, log2 partitions, exact rerun expected): one
# partition cannot hold the ~60K qualifying keys of the 1.5M-row build
@pytest.mark.parametrize("nb,np_,log2p,rerun", [(37, 1001, 0, 0), (200_000, 1_000_000, 3, 0),
                                               (1_500_000, 6_000_000, 6, 0), (1_500_000, 6_000_000, 12, 0),
                                               (1_500_000, 6_000_000, 0, 1), (0, 5000, 2, 0), (5000, 0, 2, 0)])
def test_partitioned_join_matches_oracle(engine, torch_cuda, nb, np_, log2p, rerun):
    j = dg.gen_join(nb, np_, seed=nb + np_ + log2p)
    b, p = device(torch_cuda, j)
    r = engine.join_partitioned(b, p, nb, np_, j.date_lt, j.seg_eq, log2p)
    assert tuple(r[f] for f in FIELDS) == want(j)
    assert r["mode"] == 2 and r["reruns"] == rerun


def test_partitioned_join_repeated_keys(engine, torch_cuda):
    j = dg.gen_join(300_000, 2_000_000, seed=12)
    key = j.b_key.copy()
    key[100_000:140_000] = key[:40_000]  # keys on two build rows: multiplicity 2 where both qualify
    j = dg.JoinInput(key, j.b_date, j.b_seg, j.p_fk, j.p_price, j.p_disc, dg.DATE_HI + 1, j.seg_eq, j.seed)
    b, p = device(torch_cuda, j)
    r = engine.join_partitioned(b, p, 300_000, 2_000_000, j.date_lt, j.seg_eq, 5)
    assert tuple(r[f] for f in FIELDS) == want(j) and r["reruns"] == 0


def test_partitioned_join_bad_fanout(engine, torch_cuda):
    j = dg.gen_join(1000, 1000, seed=1)
    b, p = device(torch_cuda, j)
    with pytest.raises(N.BoError) as e:
        engine.join_partitioned(b, p, 1000, 1000, j.date_lt, j.seg_eq, N.JOIN_MAX_LOG2_PARTITIONS + 1)
    assert e.value.status == -1
