"""The trained group-by sizer: q-error against the independence/uniformity
estimate it replaces, and learned-sized answers equal to the exact form's."""
import numpy as np
import pytest

from bespokeolap_artifacts_b200 import datagen as dg
from bespokeolap_artifacts_b200 import learned as L
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def trained(engine):
    x, t, naive = L.make_groupby_training_set(engine, n_tables=12, preds_per_table=30, seed=3, nb_max=2_000_000)
    rng = np.random.default_rng(1)
    idx = rng.permutation(len(x))
    tr, te = idx[: int(0.8 * len(x))], idx[int(0.8 * len(x)):]
    sizer = L.GroupBySizer(engine, seed=2)
    sizer.fit(x[tr], t[tr], epochs=3000, lr=2e-3)
    return sizer, x, t, naive, te


def test_groupby_sizer_beats_naive(trained):
    sizer, x, t, naive, te = trained
    true_groups = np.expm1(t[te, 0].astype(np.float64))
    pred = sizer.predict_host(x[te])[:, 0]
    q_mlp = L.q_error(pred, true_groups)
    q_naive = L.q_error(naive[te, 0], true_groups)
    assert np.median(q_mlp) < 1.6
    assert np.mean(np.log(q_mlp)) < np.mean(np.log(q_naive))


def test_learned_groupby_answers_equal_exact(engine, torch_cuda, trained):
    torch = torch_cuda
    sizer = trained[0]
    g = dg.gen_groupby(300_000, 4_000_000, 500_000, seed=17)
    o = O.groupby_topk(g)
    dev = engine.groupby_to_device(g)
    st = L.groupby_table_stats(engine.ctx, dev, len(g.a_ids), len(g.b_a), len(g.c_cat))
    pred = torch.zeros(2, dtype=torch.float32, device="cuda")
    sizer.predict_device(L.groupby_features(st, g.cat_set, g.year_lo, g.year_hi), pred)
    r = engine.groupby_presized(dev, g, pred)
    assert (r["n_groups"], r["keys"], r["counts"], r["min_years"]) == (
        o["n_groups"], o["keys"], o["counts"], o["min_years"])
