"""Seeded IMDB-shaped Parquet files (synthetic data) for the CEB pipelines.

Writes the 21 tables the reference's CEB loader reads
(bespoke_ceb/loader_impl.cpp:9-33).  The tables the GPU pipelines read carry
the columns those pipelines look up; the others hold one small id column
(the reference's builder is generic: it keeps whatever columns a file has,
bespoke_ceb/builder_impl.cpp:240-252).  Every value is synthetic: kinds,
roles, info types, info values and genders are codes of this module's own
vocabularies, names and titles are numbered strings.

  title       id (1..n_title, shuffled), kind_id (1..7), production_year
              (1880..2020), title; with nulls=True some kind_ids and years
              are null and a few ids repeat (in rows of equal kind and year).
  kind_type   id 1..7, kind KIND_A..KIND_G.
  role_type   id 1..12, role ROLE_A..ROLE_L.
  info_type   id 1..n_info_type (113), info INFO_TYPE_<id>.
  movie_info  movie_id (bounded Zipf over the title ids; some beyond them),
              info_type_id (skewed over 1..n_info_type + a few beyond),
              info (one of n_info_values strings V000..), note.
  cast_info   movie_id (bounded Zipf), person_id (bounded Zipf over the
              name ids), role_id (1..12); with nulls=True some null
              person_ids / role_ids.
  name        id 1..n_name (shuffled), name NAME_<id> (some in mixed case,
              some shared by two persons), gender GENDER_M / GENDER_F / null,
              name_pcode_nf (letter + 3 digits; some null with nulls=True).
  company_name id 1..n_company (shuffled), name COMP_<id> (some in mixed
              case, some shared); company_type id 1..4, kind CT_A..CT_D.
  movie_companies movie_id (bounded Zipf), company_id (bounded Zipf),
              company_type_id (1..4; some null with nulls=True).
  keyword     id 1..n_keyword, keyword KW_<id>; movie_keyword movie_id
              (bounded Zipf), keyword_id (some null with nulls=True).
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pyarrow as pa
import pyarrow.parquet as pq

KINDS = [f"KIND_{c}" for c in "ABCDEFG"]
ROLES = [f"ROLE_{c}" for c in "ABCDEFGHIJKL"]
GENDERS = ["GENDER_M", "GENDER_F"]
COMPANY_TYPES = ["CT_A", "CT_B", "CT_C", "CT_D"]
OTHER_TABLES = ["aka_name", "aka_title", "char_name", "comp_cast_type", "complete_cast", "link_type",
                "movie_info_idx", "movie_link", "person_info"]


def _zipf(rng, n: int, n_ranks: int, s: float) -> np.ndarray:
    w = np.arange(1, n_ranks + 1, dtype=np.float64) ** (-s)
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    return np.minimum(np.searchsorted(cdf, rng.random(n), side="right"), n_ranks - 1)


def _int(values: np.ndarray, null: np.ndarray | None = None) -> pa.Array:
    return pa.array(values.astype(np.int32), pa.int32(), mask=null)


def person_name(k: int) -> str:
    """NAME_<k>, every 7th in mixed case (Name_<k>), every 11th the name of
    person k // 11 (persons sharing a name)."""
    if k % 11 == 0:
        k //= 11
    return f"Name_{k:07d}" if k % 7 == 0 else f"NAME_{k:07d}"


def info_value(i: int) -> str:
    return f"V{i:03d}"


def name_pcode(k: int) -> str:
    """A short synthetic phonetic-style code per person: letter + 3 digits."""
    return f"{chr(65 + k % 26)}{(k * 7) % 1000:03d}"


def company(k: int) -> str:
    """COMP_<k>, every 5th in mixed case, every 13th sharing the name of k // 13."""
    if k % 13 == 0:
        k //= 13
    return f"Comp_{k:06d}" if k % 5 == 0 else f"COMP_{k:06d}"


def write_ceb(out: Path, n_title: int = 20_000, n_name: int = 50_000, n_cast: int = 300_000,
              n_movie_info: int = 200_000, n_info_type: int = 113, n_info_values: int = 60, seed: int = 0,
              nulls: bool = False, n_company: int = 2000, n_movie_companies: int = 60_000, n_keyword: int = 3000,
              n_movie_keyword: int = 80_000) -> Path:
    rng = np.random.default_rng(seed)
    out.mkdir(parents=True, exist_ok=True)
    # title
    tid = rng.permutation(np.arange(1, n_title + 1)).astype(np.int32)
    kind = rng.integers(1, len(KINDS) + 1, n_title)
    year = rng.integers(1880, 2021, n_title)
    kind_null = year_null = None
    if nulls:
        kind_null = rng.random(n_title) < 0.03
        year_null = rng.random(n_title) < 0.05
        # repeated ids, rows equal in kind and year (which of two rows of an id
        # the reference's unstable id sort puts last is unspecified)
        tid[-3:] = tid[:3]
        kind[-3:], year[-3:] = kind[:3], year[:3]
        kind_null[-3:], year_null[-3:] = kind_null[:3], year_null[:3]
    pq.write_table(pa.table({"id": _int(tid), "kind_id": _int(kind, kind_null),
                             "production_year": _int(year, year_null),
                             "title": [f"TITLE_{k}" for k in tid]}), out / "title.parquet")
    pq.write_table(pa.table({"id": _int(np.arange(1, len(KINDS) + 1)), "kind": KINDS}), out / "kind_type.parquet")
    pq.write_table(pa.table({"id": _int(np.arange(1, len(ROLES) + 1)), "role": ROLES}), out / "role_type.parquet")
    pq.write_table(pa.table({"id": _int(np.arange(1, n_info_type + 1)),
                             "info": [f"INFO_TYPE_{i}" for i in range(1, n_info_type + 1)]}),
                   out / "info_type.parquet")
    # name
    nid = rng.permutation(np.arange(1, n_name + 1)).astype(np.int32)
    g = rng.integers(0, 3, n_name)
    gender = pa.array([GENDERS[x] if x < 2 else None for x in g], pa.string())
    pcode_null = rng.random(n_name) < 0.02 if nulls else None
    pq.write_table(pa.table({"id": _int(nid), "name": [person_name(k) for k in nid], "gender": gender,
                             "name_pcode_nf": pa.array([name_pcode(k) for k in nid], pa.string(), mask=pcode_null)}),
                   out / "name.parquet")
    # movie_info: movie ids Zipf over titles (a few beyond the largest id)
    mi_movie = _zipf(rng, n_movie_info, n_title, 0.6) + 1
    mi_movie[rng.random(n_movie_info) < 0.002] = n_title + 5
    mi_type = _zipf(rng, n_movie_info, n_info_type, 0.8) + 1
    mi_type[rng.random(n_movie_info) < 0.002] = n_info_type + 3
    mi_info = _zipf(rng, n_movie_info, n_info_values, 0.7)
    mi_null = rng.random(n_movie_info) < 0.01 if nulls else None
    pq.write_table(pa.table({"movie_id": _int(mi_movie), "info_type_id": _int(mi_type),
                             "info": pa.array([info_value(i) for i in mi_info], pa.string(), mask=mi_null),
                             "note": pa.array([None] * n_movie_info, pa.string())}), out / "movie_info.parquet")
    # cast_info
    ci_movie = _zipf(rng, n_cast, n_title, 0.5) + 1
    ci_person = _zipf(rng, n_cast, n_name, 0.7) + 1
    ci_role = rng.integers(1, len(ROLES) + 1, n_cast)
    p_null = r_null = None
    if nulls:
        p_null = rng.random(n_cast) < 0.01
        r_null = rng.random(n_cast) < 0.01
    pq.write_table(pa.table({"movie_id": _int(ci_movie), "person_id": _int(ci_person, p_null),
                             "role_id": _int(ci_role, r_null)}), out / "cast_info.parquet")
    # companies, movie_companies, keywords, movie_keyword (a stream of their
    # own, so the tables above do not depend on these sizes)
    rng2 = np.random.default_rng([seed, 3])
    cid = rng2.permutation(np.arange(1, n_company + 1)).astype(np.int32)
    pq.write_table(pa.table({"id": _int(cid), "name": [company(k) for k in cid]}), out / "company_name.parquet")
    pq.write_table(pa.table({"id": _int(np.arange(1, len(COMPANY_TYPES) + 1)), "kind": COMPANY_TYPES}),
                   out / "company_type.parquet")
    mc_movie = _zipf(rng2, n_movie_companies, n_title, 0.5) + 1
    mc_comp = _zipf(rng2, n_movie_companies, n_company, 0.8) + 1
    mc_type = rng2.integers(1, len(COMPANY_TYPES) + 1, n_movie_companies)
    mc_null = rng2.random(n_movie_companies) < 0.01 if nulls else None
    pq.write_table(pa.table({"movie_id": _int(mc_movie), "company_id": _int(mc_comp),
                             "company_type_id": _int(mc_type, mc_null)}), out / "movie_companies.parquet")
    pq.write_table(pa.table({"id": _int(np.arange(1, n_keyword + 1)),
                             "keyword": [f"KW_{k:05d}" for k in range(1, n_keyword + 1)]}), out / "keyword.parquet")
    mk_movie = _zipf(rng2, n_movie_keyword, n_title, 0.5) + 1
    mk_kw = rng2.integers(1, n_keyword + 1, n_movie_keyword)
    mk_null = rng2.random(n_movie_keyword) < 0.01 if nulls else None
    pq.write_table(pa.table({"movie_id": _int(mk_movie), "keyword_id": _int(mk_kw, mk_null)}),
                   out / "movie_keyword.parquet")
    for t in OTHER_TABLES:
        pq.write_table(pa.table({"id": _int(np.arange(1, 4))}), out / f"{t}.parquet")
    return out
