"""GPU parity of the filtered hash join (build + probe) against the oracle and
the reference's run_q3 fixtures: match counts and fixed-point sums bit-exact,
in both the plain exact-count form and the presized form (including an
undersized prediction that must fall back to the exact rerun)."""
import json
from pathlib import Path

import numpy as np
import pytest

from bespokeolap_artifacts_b200 import datagen as dg
from bespokeolap_artifacts_b200 import native as N
from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


def same(r, o):
    return (r["build_rows"], r["match_count"], r["sum_exact"], r["sum_trunc"]) == (
        o["build_count"], o["match_count"], o["sum_exact"], o["sum_trunc"])


@pytest.mark.parametrize("nb,npr,seed", [(0, 0, 1), (1, 1, 2), (3, 10, 3), (1000, 4003, 4), (20_000, 80_001, 5),
                                         (1_500_000, 6_000_000, 6)])
def test_join_plain_matches_oracle(engine, nb, npr, seed):
    j = dg.gen_join(nb, npr, seed)
    r = engine.join_host(j, mode=0)
    assert same(r, O.join_agg(j))
    assert r["overflowed"] == 0 and r["reruns"] == 0


@pytest.mark.parametrize("pred_scale", [1.0, 0.5, 3.0])
def test_join_presized_matches_oracle(engine, pred_scale):
    j = dg.gen_join(200_000, 800_000, 7)
    o = O.join_agg(j)
    r = engine.join_host(j, mode=1, predicted_rows=o["build_count"] * pred_scale)
    assert same(r, o)
    assert r["reruns"] == 0


def test_join_underpredicted_falls_back_exactly(engine):
    j = dg.gen_join(200_000, 800_000, 8)
    o = O.join_agg(j)
    r = engine.join_host(j, mode=1, predicted_rows=10.0)  # far too small: table overflows
    assert r["reruns"] == 1
    assert same(r, o)


@pytest.mark.parametrize("case", json.loads((GOLDEN / "q3_reference.json").read_text()),
                         ids=lambda c: f"seed{c['seed']}")
def test_join_matches_reference_q3_golden(engine, case):
    j = dg.gen_join(case["n_build"], case["n_probe"], case["seed"])
    r = engine.join_host(j, mode=0)
    assert r["sum_trunc"] == case["revenue_sum"]
    assert r["match_count"] == case["lineitems_emitted"]


def test_join_duplicate_build_keys(engine):
    j = dg.gen_join(50_000, 200_000, 9)
    j.b_key[1::2] = j.b_key[0::2][: len(j.b_key[1::2])]  # every key twice -> multiplicity 2
    o = O.join_agg(j)
    assert same(engine.join_host(j, mode=0), o)
    assert same(engine.join_host(j, mode=1, predicted_rows=o["build_count"]), o)


def test_join_no_qualifying_rows(engine):
    j = dg.gen_join(10_000, 40_000, 10, date_lt=dg.DATE_LO)  # date < DATE_LO never holds
    r = engine.join_host(j, mode=0)
    assert r["build_rows"] == 0 and r["match_count"] == 0 and r["sum_exact"] == 0


def test_join_device_presized_repeatable(engine, torch_cuda):
    """The asynchronous presized form leaves the context clean for the next call."""
    torch = torch_cuda
    j = dg.gen_join(100_000, 400_000, 11)
    o = O.join_agg(j)
    build = [torch.from_numpy(x).cuda() for x in (j.b_key, j.b_date, j.b_seg)]
    probe = [torch.from_numpy(x).cuda() for x in (j.p_fk, j.p_price, j.p_disc)]
    pred = torch.tensor([float(o["build_count"])], dtype=torch.float32, device="cuda")
    for _ in range(3):
        r = engine.join_presized(build, probe, j.n_build, j.n_probe, j.date_lt, j.seg_eq, pred)
        assert same(r, o)
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    engine.join_count_device(build, j.n_build, j.date_lt, j.seg_eq, cnt)
    engine.synchronize()
    assert int(cnt.item()) == o["build_count"]


def test_join_value_out_of_contract(engine):
    j = dg.gen_join(1000, 4000, 12)
    o = O.join_agg(j)
    if o["match_count"] == 0:
        pytest.skip("no matches")
    q = (j.b_date < j.date_lt) & (j.b_seg == j.seg_eq)
    k = j.b_key[q][0]
    i = int(np.nonzero(j.p_fk == k)[0][0]) if (j.p_fk == k).any() else None
    if i is None:
        j.p_fk[0] = k
        i = 0
    j.p_disc[i] = 300
    with pytest.raises(N.BoError) as e:
        engine.join_host(j, mode=0)
    assert e.value.status == -6
