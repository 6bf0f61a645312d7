"""CEB query 1a on the GPU (bo_ceb_q1a through the C ABI) against the
reference's own CEB engine (compiled unchanged into
oracle/_ref/ref_ceb_driver) on the same seeded IMDB-shaped Parquet files,
with and without nulls, and at a larger size against the restatement: the
counts must be equal."""
from pathlib import Path

import pytest

from bespokeolap_artifacts_b200 import ceb
from bespokeolap_artifacts_b200.ceb_data import write_ceb
from ceb_restate import q1a as q1a_restated
from test_ceb_cpu import Q1A_CASES, REF_CEB, reference, request

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nulls,seed", [(False, 1), (True, 2), (True, 3)])
def test_q1a_gpu_matches_reference(engine, torch_cuda, tmp_path, nulls, seed):
    if not REF_CEB.exists():
        pytest.skip("reference CEB driver not built")
    data = write_ceb(tmp_path / "d", n_title=4000, n_name=8000, n_cast=40_000, n_movie_info=30_000, seed=seed,
                     nulls=nulls)
    tables = ceb.load_tables(data)
    got = reference(data, tmp_path / "ref", [request(c) for c in Q1A_CASES])
    for case, g in zip(Q1A_CASES, got):
        assert ceb.q1a(engine, tables, *case) == int(g[1][0]), case


def test_q1a_gpu_larger_tables(engine, torch_cuda, tmp_path):
    data = write_ceb(tmp_path / "d", n_title=200_000, n_name=400_000, n_cast=3_000_000, n_movie_info=1_500_000,
                     seed=5, nulls=True)
    tables = ceb.load_tables(data)
    for case in Q1A_CASES[:3]:
        assert ceb.q1a(engine, tables, *case) == q1a_restated(data, *case), case


def test_q1a_gpu_empty_title(engine, torch_cuda, tmp_path):
    data = write_ceb(tmp_path / "d", n_title=100, n_name=100, n_cast=1000, n_movie_info=1000, seed=6)
    tables = ceb.load_tables(data)
    case = list(Q1A_CASES[0])
    case[7], case[8] = "1000", "3000"  # no production year in range: no title row qualifies
    assert ceb.q1a(engine, tables, *case) == 0


def test_builder_order_on_gpu(engine, torch_cuda, tmp_path):
    """cast_info by (movie_id, role_id) and movie_info by (movie_id,
    info_type_id), as the reference builder orders them: the device columns
    come out in numpy's stable lexicographic order of the stored values (0
    where null), every column moved with its row, and q1a's count is
    unchanged."""
    import numpy as np
    import pyarrow.parquet as pq

    data = write_ceb(tmp_path / "d", n_title=3000, n_name=6000, n_cast=500_000, n_movie_info=200_000, seed=7,
                     nulls=True)
    tables = ceb.load_tables(data)
    before = ceb.q1a(engine, tables, *Q1A_CASES[0])
    ceb.builder_order(engine, tables)
    for table, (p, s) in (("cast_info", ("movie_id", "role_id")), ("movie_info", ("movie_id", "info_type_id"))):
        raw = pq.read_table(data / f"{table}.parquet")
        loaded = [c for c in raw.column_names if c in tables.tables[table]]
        ints = {c: np.nan_to_num(raw[c].to_numpy(zero_copy_only=False)).astype(np.int64) for c in loaded
                if tables.col(table, c).dictionary is None}
        order = np.lexsort((ints[s], ints[p]))  # stable: ties keep the input order
        for c in loaded:
            col = tables.col(table, c)
            dev = col.values.cpu().numpy()
            if col.dictionary is None:
                assert np.array_equal(dev, ints[c][order]), (table, c)
            else:  # string column: the codes decode to the input strings in the new order
                want = raw[c].to_pylist()
                nl = col.is_null.cpu().numpy() if col.is_null is not None else np.zeros(len(dev), np.uint8)
                got = [None if nl[i] else col.dictionary[dev[i]] for i in range(len(dev))]
                assert got == [want[i] for i in order], (table, c)
        nl = tables.col(table, "movie_id").is_null
        assert nl is None or not nl.any().item()
    assert ceb.q1a(engine, tables, *Q1A_CASES[0]) == before


def gpu_q10a_rows(engine, tables, case):
    rows = ceb.q10a(engine, tables, *case)
    return sorted((n, v, lo, hi) for n, v, _, lo, hi in rows)


@pytest.mark.parametrize("nulls,seed", [(False, 1), (True, 2)])
def test_q10a_gpu_matches_reference(engine, torch_cuda, tmp_path, nulls, seed):
    """CEB query 10a: the GPU's (name, info, min, max) rows equal the
    reference engine's as sets (the reference emits them in its aggregation
    order); the dense-matrix aggregation runs here."""
    if not REF_CEB.exists():
        pytest.skip("reference CEB driver not built")
    from test_ceb_cpu import Q10A_CASES, q10a_csv_rows, request10a

    data = write_ceb(tmp_path / "d", n_title=4000, n_name=8000, n_cast=40_000, n_movie_info=30_000, seed=seed,
                     nulls=nulls)
    tables = ceb.load_tables(data, ceb.Q10A_COLUMNS)
    got = reference(data, tmp_path / "ref", [request10a(c) for c in Q10A_CASES])
    for case, g in zip(Q10A_CASES, got):
        assert gpu_q10a_rows(engine, tables, case) == q10a_csv_rows(g), case


def test_q10a_gpu_hash_aggregation(engine, torch_cuda, tmp_path):
    """More name strings x info values than the dense matrix holds: the hash
    aggregation runs and agrees with the restatement."""
    from bespokeolap_artifacts_b200.ceb import string_pool
    from ceb_restate import q10a as q10a_restated

    data = write_ceb(tmp_path / "d", n_title=100_000, n_name=700_000, n_cast=2_000_000, n_movie_info=600_000,
                     seed=8, nulls=True)
    tables = ceb.load_tables(data, ceb.Q10A_COLUMNS)
    pool = string_pool(data)
    infos = [f"V{i:03d}" for i in range(10)]
    case = (["1", "2", "3", "4", "5"], infos, "%1%", ["KIND_A", "KIND_B", "KIND_C"], ["ROLE_A", "ROLE_B", "ROLE_C"])
    got = gpu_q10a_rows(engine, tables, case)
    assert not ceb.q10a.last_dense
    assert got == q10a_restated(data, *case, pool)
    assert len(got) > 1000


@pytest.mark.parametrize("nulls,seed", [(False, 1), (True, 2)])
def test_q3b_gpu_matches_reference(engine, torch_cuda, tmp_path, nulls, seed):
    """CEB query 3b: the GPU's rows equal the reference engine's, in its
    order (count desc, then title, name, company)."""
    if not REF_CEB.exists():
        pytest.skip("reference CEB driver not built")
    from test_ceb_cpu import Q3B_CASES, q3b_csv_rows, request3b

    data = write_ceb(tmp_path / "d", n_title=4000, n_name=8000, n_cast=40_000, n_movie_info=30_000, seed=seed,
                     nulls=nulls, n_company=500, n_movie_companies=12_000, n_keyword=800, n_movie_keyword=15_000)
    tables = ceb.load_tables(data, ceb.Q3B_COLUMNS)
    ceb.builder_order(engine, tables)
    got = reference(data, tmp_path / "ref", [request3b(c) for c in Q3B_CASES])
    for case, g in zip(Q3B_CASES, got):
        assert ceb.q3b(engine, tables, *case) == q3b_csv_rows(g), case


def test_q3b_gpu_larger_tables(engine, torch_cuda, tmp_path):
    from ceb_restate import q3b as q3b_restated

    data = write_ceb(tmp_path / "d", n_title=100_000, n_name=200_000, n_cast=1_500_000, n_movie_info=1000, seed=9,
                     nulls=True, n_company=20_000, n_movie_companies=400_000, n_keyword=5000,
                     n_movie_keyword=500_000)
    tables = ceb.load_tables(data, ceb.Q3B_COLUMNS)
    case = ("%1%", "a%", "%00%", ["KIND_A", "KIND_B", "KIND_C"], ["ROLE_A", "ROLE_B", "ROLE_C"])
    got = ceb.q3b(engine, tables, *case)
    assert got == q3b_restated(data, *case)
    assert len(got) > 100
