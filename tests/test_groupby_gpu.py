"""GPU parity of the skewed three-way join + group-by + onesweep radix sort +
top-k against the oracle (which restates the reference's dense-count, min and
LSD-ordering patterns): bit-exact counts, min years, keys and order."""
import numpy as np
import pytest

from bespokeolap_artifacts_b200 import datagen as dg
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def same(r, o):
    return (r["n_groups"], r["joined_rows"], r["keys"], r["counts"], r["min_years"]) == (
        o["n_groups"], o["joined_rows"], o["keys"], o["counts"], o["min_years"])


@pytest.mark.parametrize("n", [0, 1, 7, 4095, 4096, 4097, 100_003, 1_000_000])
def test_radix_sort_matches_oracle(engine, n):
    rng = np.random.default_rng(n)
    k = rng.integers(0, 2**64, size=n, dtype=np.uint64)
    if n > 10:
        k[::5] = k[3]  # ties: stability matters
    v = np.arange(n, dtype=np.uint32)
    gk, gv = engine.radix_sort_pairs_host(k, v)
    ok, ov = O.radix_sort_pairs(k, v)
    assert np.array_equal(gk, ok) and np.array_equal(gv, ov)


@pytest.mark.parametrize("bits", [(0, 8), (0, 24), (16, 40), (0, 48)])
def test_radix_sort_bit_ranges(engine, bits):
    lo, hi = bits
    rng = np.random.default_rng(hi)
    n = 200_001
    k = rng.integers(0, 2**hi, size=n, dtype=np.uint64) & ~np.uint64((1 << lo) - 1)
    v = np.arange(n, dtype=np.uint32)
    gk, gv = engine.radix_sort_pairs_host(k, v, lo, hi)
    order = np.argsort(k, kind="stable")
    assert np.array_equal(gk, k[order]) and np.array_equal(gv, v[order])


@pytest.mark.parametrize("sizes,seed", [((1000, 20_000, 5000), 1), ((20_000, 300_000, 40_000), 2),
                                        ((2_500_000, 36_000_000, 4_000_000), 3)])
def test_groupby_plain_matches_oracle(engine, sizes, seed):
    g = dg.gen_groupby(*sizes, seed=seed)
    o = O.groupby_topk(g)
    dev = engine.groupby_to_device(g)
    r = engine.groupby_plain(dev, g)
    assert same(r, o), (r, o)
    assert r["exact_distinct"] == o["n_groups"]


@pytest.mark.parametrize("scale", [1.0, 0.6, 4.0])
def test_groupby_presized_matches_oracle(engine, torch_cuda, scale):
    torch = torch_cuda
    g = dg.gen_groupby(200_000, 3_000_000, 400_000, seed=4)
    o = O.groupby_topk(g)
    dev = engine.groupby_to_device(g)
    pred = torch.tensor([o["n_groups"] * scale], dtype=torch.float32, device="cuda")
    r = engine.groupby_presized(dev, g, pred)
    assert same(r, o)
    assert r["reruns"] == 0


def test_groupby_underpredicted_falls_back(engine, torch_cuda):
    torch = torch_cuda
    g = dg.gen_groupby(200_000, 3_000_000, 400_000, seed=5)
    o = O.groupby_topk(g)
    dev = engine.groupby_to_device(g)
    pred = torch.tensor([5.0], dtype=torch.float32, device="cuda")
    r = engine.groupby_presized(dev, g, pred)
    assert r["reruns"] == 1
    assert same(r, o)


def test_groupby_no_qualifying_rows(engine, torch_cuda):
    g = dg.gen_groupby(1000, 50_000, 5000, seed=6, year_lo=3000, year_hi=3001)
    o = O.groupby_topk(g)
    r = engine.groupby_plain(engine.groupby_to_device(g), g)
    assert o["n_groups"] == 0 and r["n_groups"] == 0 and r["keys"] == []


def test_groupby_out_of_range_ids_are_dropped(engine):
    g = dg.gen_groupby(5000, 100_000, 20_000, seed=7)
    g.b_c[::97] = -3             # negative c_id: dropped
    g.b_c[1::89] = len(g.c_cat) + 5  # past C: dropped
    g.b_a[2::83] = 10 ** 8       # not an id of A: dropped
    o = O.groupby_topk(g)
    r = engine.groupby_plain(engine.groupby_to_device(g), g)
    assert same(r, o)


def test_groupby_distinct_prepass(engine, torch_cuda):
    torch = torch_cuda
    g = dg.gen_groupby(50_000, 800_000, 100_000, seed=8)
    o = O.groupby_topk(g)
    out = torch.zeros(2, dtype=torch.int64, device="cuda")
    engine.groupby_distinct_device(engine.groupby_to_device(g), g, out)
    engine.synchronize()
    assert out.tolist() == [o["n_groups"], o["joined_rows"]]


def test_groupby_prebuilt_a_mask(engine, torch_cuda):
    torch = torch_cuda
    g = dg.gen_groupby(100_000, 1_500_000, 200_000, seed=9)
    o = O.groupby_topk(g)
    dev = engine.groupby_to_device(g, prebuild_a_mask=True)
    assert same(engine.groupby_plain(dev, g), o)
    pred = torch.tensor([float(o["n_groups"])], dtype=torch.float32, device="cuda")
    assert same(engine.groupby_presized(dev, g, pred), o)
