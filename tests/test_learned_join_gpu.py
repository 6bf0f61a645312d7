"""The trained sizer: sketches on the GPU, training pairs from the plain GPU
pipeline, q-error against the independence estimate it replaces, and the
learned-sized join's answers equal to the exact form's."""
import numpy as np
import pytest

from bespokeolap_artifacts_b200 import datagen as dg
from bespokeolap_artifacts_b200 import learned as L
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_sketch_matches_numpy(engine, torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(3)
    v = rng.integers(-5000, 90000, size=300_001, dtype=np.int32)
    s = L.sketch_i32(engine.ctx, torch.from_numpy(v).cuda(), len(v))
    assert (s.min, s.max, s.n) == (int(v.min()), int(v.max()), len(v))
    span = s.max - s.min + 1
    bins = ((v.astype(np.int64) - s.min) * 64) // span
    assert np.array_equal(s.hist, np.bincount(bins, minlength=64))
    true_d = len(np.unique(v))
    assert abs(s.distinct - true_d) / true_d < 0.05  # HLL with 4096 registers: ~1.6% std error
    seg = rng.integers(0, 7, size=100_003, dtype=np.uint8)
    h = L.histogram_small(engine.ctx, torch.from_numpy(seg).cuda(), 1, len(seg), 256)
    assert np.array_equal(h, np.bincount(seg, minlength=256))


@pytest.fixture(scope="module")
def trained(engine):
    x, t, naive = L.make_join_training_set(engine, n_tables=20, preds_per_table=40, seed=99, n_max=800_000)
    rng = np.random.default_rng(0)
    idx = rng.permutation(len(x))
    tr, te = idx[: int(0.8 * len(x))], idx[int(0.8 * len(x)):]
    sizer = L.JoinSizer(engine, seed=5)
    sizer.fit(x[tr], t[tr], epochs=3000, lr=2e-3)
    return sizer, x, t, naive, te


def test_sizer_beats_independence_estimate(trained):
    sizer, x, t, naive, te = trained
    true = np.expm1(t[te, 0].astype(np.float64))
    q_mlp = L.q_error(sizer.predict_host(x[te]), true)
    q_naive = L.q_error(naive[te], true)
    assert np.median(q_mlp) < 1.5
    assert np.percentile(q_mlp, 90) < np.percentile(q_naive, 90)
    assert np.mean(np.log(q_mlp)) < np.mean(np.log(q_naive))


def test_learned_join_answers_equal_exact(engine, torch_cuda, trained):
    torch = torch_cuda
    sizer = trained[0]
    j = dg.gen_join(400_000, 1_600_000, 21)
    o = O.join_agg(j)
    b = [torch.from_numpy(a).cuda() for a in (j.b_key, j.b_date, j.b_seg)]
    p = [torch.from_numpy(a).cuda() for a in (j.p_fk, j.p_price, j.p_disc)]
    st = L.join_table_stats(engine.ctx, b[0], b[1], b[2], j.n_build)
    pred = torch.zeros(1, dtype=torch.float32, device="cuda")
    sizer.predict_device(L.join_features(st, j.date_lt, j.seg_eq), pred)
    r = engine.join_presized(b, p, j.n_build, j.n_probe, j.date_lt, j.seg_eq, pred)
    assert (r["build_rows"], r["match_count"], r["sum_exact"], r["sum_trunc"]) == (
        o["build_count"], o["match_count"], o["sum_exact"], o["sum_trunc"])
