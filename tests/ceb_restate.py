"""A plain-Python restatement of CEB query 1a (run_q1a,
bespoke_ceb/query_q1a.cpp:155-655) over the Parquet files, for the tests:
the reference's id masks, null skips, dense per-movie counts and the
factorised sum over the qualifying title rows."""
from __future__ import annotations

from pathlib import Path

import pyarrow.parquet as pq

from bespokeolap_artifacts_b200.ceb import NULL_WORDS, stoi


def _cols(path: Path, table: str, names):
    t = pq.read_table(Path(path) / f"{table}.parquet", columns=list(names))
    return [t[n].to_pylist() for n in names], t.num_rows


def _dim_mask(path, table, str_col, allowed):
    (ids, vals), n = _cols(path, table, ("id", str_col))
    allowed = {v for v in allowed if v not in NULL_WORDS}
    return {i for i, v in zip(ids, vals) if i is not None and v is not None and i >= 0 and v in allowed}


def q1a(path, id1, id2, info1, info2, kind, role, gender, year1, year2) -> int:
    y1, y2 = stoi(year1), stoi(year2)
    kinds = _dim_mask(path, "kind_type", "kind", kind)
    roles = _dim_mask(path, "role_type", "role", role)
    persons = _dim_mask(path, "name", "gender", gender)
    (it_ids,), n_it = _cols(path, "info_type", ("id",))
    size = max([n_it + 1] + [i + 1 for i in it_ids if i is not None and i >= 0])
    f1 = {i for i in (stoi(v) for v in id1 if v not in NULL_WORDS) if i is not None and 0 <= i < size}
    f2 = {i for i in (stoi(v) for v in id2 if v not in NULL_WORDS) if i is not None and 0 <= i < size}
    v1 = {v for v in info1 if v not in NULL_WORDS}
    v2 = {v for v in info2 if v not in NULL_WORDS}
    (tid, tkind, tyear), _ = _cols(path, "title", ("id", "kind_id", "production_year"))
    movies = [m for m, k, y in zip(tid, tkind, tyear)
              if m is not None and k is not None and y is not None and m >= 0 and y2 <= y <= y1 and k in kinds]
    if not movies:
        return 0
    mx = max(movies)
    (mm, mt, mi), _ = _cols(path, "movie_info", ("movie_id", "info_type_id", "info"))
    c1, c2 = {}, {}
    for m, ty, v in zip(mm, mt, mi):
        if ty is None or v is None or m is None or m < 0 or m > mx:
            continue
        if ty in f1 and v in v1:
            c1[m] = c1.get(m, 0) + 1
        if ty in f2 and v in v2:
            c2[m] = c2.get(m, 0) + 1
    both = {m for m in movies if c1.get(m) and c2.get(m)}
    (cm, cp, cr), _ = _cols(path, "cast_info", ("movie_id", "person_id", "role_id"))
    cast = {}
    for m, p, r in zip(cm, cp, cr):
        if m is None or p is None or r is None or m not in both or r not in roles or p not in persons:
            continue
        cast[m] = cast.get(m, 0) + 1
    return sum(cast.get(m, 0) * c1.get(m, 0) * c2.get(m, 0) for m in movies)
