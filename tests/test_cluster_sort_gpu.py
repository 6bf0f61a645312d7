"""The one-launch cluster sort (pairs held in the distributed shared memory of
1 to 16 CTAs, about 1K pairs per CTA; up to 131,072 pairs where the device
schedules a 16-CTA cluster, else 65,536) against the oracle's stable LSD sort
and numpy's stable argsort: sizes at every cluster-size boundary, ties
(stability across CTAs), bit ranges, and digits that every key shares
(skipped passes).  Above the limit the onesweep passes sort again."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [2, 3, 511, 1024, 1025, 2049, 4097, 8191, 8192, 8193, 16384, 16385, 32768, 32769,
                               65535, 65536, 65537, 131072, 131073])
def test_cluster_sort_sizes_match_oracle(engine, n):
    rng = np.random.default_rng(n)
    k = rng.integers(0, 2**64, size=n, dtype=np.uint64)
    k[::3] = k[1]  # a third of the keys tie: their input order must survive every pass
    v = np.arange(n, dtype=np.uint32)
    gk, gv = engine.radix_sort_pairs_host(k, v)
    ok, ov = O.radix_sort_pairs(k, v)
    assert np.array_equal(gk, ok) and np.array_equal(gv, ov)


@pytest.mark.parametrize("n,bits", [(5000, (0, 8)), (30_000, (0, 20)), (60_000, (16, 40)), (20_000, (0, 64)),
                                    (12_000, (8, 13))])
def test_cluster_sort_bit_ranges(engine, n, bits):
    lo, hi = bits
    rng = np.random.default_rng(n + hi)
    k = rng.integers(0, 2**63, size=n, dtype=np.uint64)
    v = rng.permutation(n).astype(np.uint32)
    gk, gv = engine.radix_sort_pairs_host(k, v, lo, hi)
    field = (k >> np.uint64(lo)) & np.uint64((1 << (hi - lo)) - 1) if hi - lo < 64 else k
    order = np.argsort(field, kind="stable")
    assert np.array_equal(gk, k[order]) and np.array_equal(gv, v[order])


def test_cluster_sort_shared_digits_are_skipped_correctly(engine):
    """Keys that differ only in bits 24..31 (every other digit is the same for
    all keys: those passes move nothing) across 4 CTAs."""
    n = 30_001
    rng = np.random.default_rng(5)
    k = (np.uint64(0xABCD00000077) | (rng.integers(0, 256, size=n, dtype=np.uint64) << np.uint64(24)))
    v = np.arange(n, dtype=np.uint32)
    gk, gv = engine.radix_sort_pairs_host(k, v, 0, 64)
    order = np.argsort(k, kind="stable")
    assert np.array_equal(gk, k[order]) and np.array_equal(gv, v[order])
