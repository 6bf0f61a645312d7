"""The learned join in one call (bo_join_learned*): its fused prediction +
init kernel must size the table exactly as bo_mlp_predict_counts followed by
bo_join_presized_device does (same prediction, bit for bit; same capacity;
same result record), and the host form must give the oracle's answer -- the
restated filtered join of run_q3 (bespoke_tpch/query_q3.cpp:182-260) --
whether the prediction is adequate or far too low (exact rerun)."""
import ctypes as C

import numpy as np
import pytest

from bespokeolap_artifacts_b200 import datagen as dg
from bespokeolap_artifacts_b200 import learned as L
from bespokeolap_artifacts_b200 import native as N
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FIELDS = ("build_rows", "match_count", "sum_exact", "sum_trunc")


def device(torch, j):
    b = [torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (j.b_key, j.b_date, j.b_seg)]
    p = [torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (j.p_fk, j.p_price, j.p_disc)]
    return b, p


def sizer_predicting(engine, rows: float, seed: int = 3) -> L.JoinSizer:
    """A sizer whose output is log1p(rows) for every input (weights of the
    last layer zero, its bias set), plus small random hidden weights."""
    s = L.JoinSizer(engine, seed=seed)
    prm = s.mlp.get_params()
    lay = L.JOIN_FEATURES * 64 + 64 + 2 * (64 * 64 + 64)  # offset of the output layer
    prm[lay:lay + 64] = 0.0
    prm[-1] = np.float32(np.log1p(rows))
    s.mlp.set_params(prm)
    return s


@pytest.mark.parametrize("rows_factor", [1.0, 3.0])
def test_fused_matches_two_calls(engine, torch_cuda, rows_factor):
    torch = torch_cuda
    j = dg.gen_join(1_500_000, 6_000_000, seed=5)
    exact = O.join_agg(j)["build_count"]
    s = sizer_predicting(engine, exact * rows_factor)
    b, p = device(torch, j)
    feats = np.linspace(0.0, 1.0, L.JOIN_FEATURES).astype(np.float32)
    sz = C.sizeof(N.JoinResult)
    out_a = torch.zeros(sz, dtype=torch.uint8, device="cuda")
    out_b = torch.zeros(sz, dtype=torch.uint8, device="cuda")
    pred_a = torch.zeros(1, dtype=torch.float32, device="cuda")
    pred_b = torch.zeros(1, dtype=torch.float32, device="cuda")
    s.join_device(feats, b, p, j.n_build, j.n_probe, j.date_lt, j.seg_eq, out_a, pred_a)
    s.predict_device(feats, pred_b)
    engine.join_presized_device(b, p, j.n_build, j.n_probe, j.date_lt, j.seg_eq, pred_b, out_b)
    engine.synchronize()
    assert pred_a.cpu().numpy().tobytes() == pred_b.cpu().numpy().tobytes()
    ra = N.JoinResult.from_buffer_copy(out_a.cpu().numpy().tobytes()).as_dict()
    rb = N.JoinResult.from_buffer_copy(out_b.cpu().numpy().tobytes()).as_dict()
    assert ra == rb and ra["overflowed"] == 0
    o = O.join_agg(j)
    assert (ra["build_rows"], ra["match_count"], ra["sum_exact"], ra["sum_trunc"]) == (
        o["build_count"], o["match_count"], o["sum_exact"], o["sum_trunc"])


def test_host_form_reruns_on_low_prediction(engine, torch_cuda):
    j = dg.gen_join(1_500_000, 6_000_000, seed=6)
    s = sizer_predicting(engine, 10.0)
    b, p = device(torch_cuda, j)
    r = s.join(np.zeros(L.JOIN_FEATURES, np.float32), b, p, j.n_build, j.n_probe, j.date_lt, j.seg_eq)
    o = O.join_agg(j)
    assert (r["build_rows"], r["match_count"], r["sum_exact"], r["sum_trunc"]) == (
        o["build_count"], o["match_count"], o["sum_exact"], o["sum_trunc"])
    assert r["reruns"] == 1
