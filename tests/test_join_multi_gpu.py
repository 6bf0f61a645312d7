"""Shared joins (bo_join_multi_*): many filtered joins of the same build and
probe tables in one pass each must give every query exactly the result of the
solo filtered join (the oracle's restatement of run_q3's filtered join,
bespoke_tpch/query_q3.cpp:182-260): one query, many, the maximum of 32,
repeated and identical predicates, queries no row qualifies for, empty
sides, and repeated build keys (exact solo reruns)."""
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


def oracle_answers(j, params):
    out = []
    for d, s in params:
        jj = dg.JoinInput(j.b_key, j.b_date, j.b_seg, j.p_fk, j.p_price, j.p_disc, d, s, j.seed)
        r = O.join_agg(jj)
        distinct = len(np.unique(j.b_key[(j.b_date < d) & (j.b_seg == s)]))
        out.append((r["build_count"], distinct, r["match_count"], r["sum_exact"], r["sum_trunc"]))
    return out


def params_for(n, seed):
    rng = np.random.default_rng(seed)
    return [(int(rng.integers(dg.DATE_LO, dg.DATE_HI + 2)), int(rng.integers(0, 6))) for _ in range(n)]


@pytest.mark.parametrize("nb,np_,nq", [(200_000, 1_000_000, 1), (200_000, 1_000_000, 7), (1_500_000, 6_000_000, 32),
                                        (37, 1001, 5), (0, 5000, 3), (5000, 0, 4)])
def test_join_multi_matches_oracle(engine, torch_cuda, nb, np_, nq):
    j = dg.gen_join(nb, np_, seed=nb + np_ + nq)
    params = params_for(nq, nb + nq)
    params[-1] = params[0]            # a repeated query
    if nq > 2:
        params[1] = (dg.DATE_LO, 0)   # no row has date < DATE_LO
    b, p = device(torch_cuda, j)
    got = engine.join_multi(b, p, nb, np_, params)
    want = oracle_answers(j, params)
    for g, w in zip(got, want):
        assert tuple(g[f] for f in FIELDS) == w
        assert g["reruns"] == 0 and g["overflowed"] == 0


def test_join_multi_repeated_keys_rerun_exactly(engine, torch_cuda):
    j = dg.gen_join(100_000, 400_000, seed=9)
    key = j.b_key.copy()
    key[50_000:50_100] = key[:100]    # keys that appear twice
    j = dg.JoinInput(key, j.b_date, j.b_seg, j.p_fk, j.p_price, j.p_disc, j.date_lt, j.seg_eq, j.seed)
    params = [(dg.DATE_HI + 1, s) for s in range(5)] + params_for(4, 2)
    b, p = device(torch_cuda, j)
    got = engine.join_multi(b, p, 100_000, 400_000, params)
    want = oracle_answers(j, params)
    for g, w in zip(got, want):
        assert tuple(g[f] for f in FIELDS) == w
        assert g["reruns"] == 1


def test_join_multi_device_async_and_limits(engine, torch_cuda):
    torch = torch_cuda
    j = dg.gen_join(50_000, 200_000, seed=4)
    params = params_for(3, 8)
    b, p = device(torch, j)
    out = torch.zeros(3 * C_sizeof(), dtype=torch.uint8, device="cuda")
    engine.join_multi_device(b, p, 50_000, 200_000, params, out)
    engine.synchronize()
    host = out.cpu().numpy().tobytes()
    for i, w in enumerate(oracle_answers(j, params)):
        r = N.JoinResult.from_buffer_copy(host[i * C_sizeof():(i + 1) * C_sizeof()]).as_dict()
        assert tuple(r[f] for f in FIELDS) == w
    for bad in ([], params_for(N.JOIN_MULTI_MAX + 1, 1), [(0, 256)]):
        with pytest.raises(N.BoError) as e:
            engine.join_multi(b, p, 50_000, 200_000, bad) if bad else engine.ctx.call(
                "bo_join_multi_host", None, None, None, 0, None)
        assert e.value.status == -1


def C_sizeof():
    import ctypes
    return ctypes.sizeof(N.JoinResult)
