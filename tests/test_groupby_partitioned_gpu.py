"""The radix-partitioned group-by (bo_groupby_topk_partitioned*) gives the
oracle's answer bit-exactly -- the restated dense-count / min / LSD-ordering
patterns (bespoke_ceb/query_q1a.cpp, query_q10a.cpp:843-856,
bespoke_tpch/query_q10.cpp:318-372) -- at every fan-out, with Zipf heavy
hitters, with a joined-rows prediction far too low, and with more groups than
one partition's shared table holds (exact plain rerun)."""
import numpy as np
import pytest

from bespokeolap_artifacts_b200 import datagen as dg
from bespokeolap_artifacts_b200 import learned as L
from bespokeolap_artifacts_b200 import native as N
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def same(r, o):
    return (r["n_groups"], r["joined_rows"], r["keys"], r["counts"], r["min_years"]) == (
        o["n_groups"], o["joined_rows"], o["keys"], o["counts"], o["min_years"])


# (sizes, seed, log2 partitions, exact rerun expected): one partition cannot
# hold the ~10^5 groups of the full-size case (its shared table has 8192
# slots), so that call reruns exactly -- the fan-out rule never picks it.
@pytest.mark.parametrize("sizes,seed,log2p,rerun", [((1000, 20_000, 5000), 1, 0, 0), ((20_000, 300_000, 40_000), 2, 3, 0),
                                                     ((2_500_000, 36_000_000, 4_000_000), 3, 0, 1),
                                                     ((2_500_000, 36_000_000, 4_000_000), 3, 6, 0),
                                                     ((2_500_000, 36_000_000, 4_000_000), 3, 12, 0)])
def test_partitioned_matches_oracle(engine, sizes, seed, log2p, rerun):
    g = dg.gen_groupby(*sizes, seed=seed)
    o = O.groupby_topk(g)
    dev = engine.groupby_to_device(g)
    r = engine.groupby_partitioned(dev, g, log2p, predicted_joined_rows=float(o["joined_rows"]))
    assert same(r, o), (r, o)
    assert r["mode"] == 2 and r["reruns"] == rerun


def test_partitioned_many_groups_and_flat_keys(engine):
    # nearly every C row qualifies and a_id is close to uniform over 3M ids:
    # ~2M groups, far more than one partition's 8192-slot table at low fan-out
    g = dg.gen_groupby(3_000_000, 8_000_000, 100_000, seed=5, s_a=0.2, s_c=0.2, n_cat_set=64,
                       year_lo=1900, year_hi=2020)
    o = O.groupby_topk(g)
    dev = engine.groupby_to_device(g)
    log2p = L.GroupBySizer.fanout(o["n_groups"], l2_bytes=16 << 20)
    assert log2p >= 8
    r = engine.groupby_partitioned(dev, g, log2p, predicted_joined_rows=float(o["joined_rows"]))
    assert same(r, o) and r["reruns"] == 0
    r = engine.groupby_partitioned(dev, g, 2, predicted_joined_rows=float(o["joined_rows"]))
    assert same(r, o) and r["reruns"] == 1  # 4 partitions of ~500K groups overflow their tables


def test_partitioned_ignores_low_joined_prediction(engine):
    # the record buffers take the one-record-per-B-row bound at this size, so
    # a far too low joined-rows prediction cannot make the call rerun
    g = dg.gen_groupby(50_000, 4_000_000, 40_000, seed=6, n_cat_set=40)
    o = O.groupby_topk(g)
    dev = engine.groupby_to_device(g)
    r = engine.groupby_partitioned(dev, g, 5, predicted_joined_rows=1.0)
    assert same(r, o) and r["reruns"] == 0 and r["mode"] == 2


def test_partitioned_bad_fanout(engine):
    g = dg.gen_groupby(1000, 20_000, 5000, seed=1)
    dev = engine.groupby_to_device(g)
    with pytest.raises(N.BoError) as e:
        engine.groupby_partitioned(dev, g, N.GB_MAX_LOG2_PARTITIONS + 1, 1000.0)
    assert e.value.status == -1
