"""CEB tables on the device in the reference's column layout, and the CEB
pipelines that run on them.

The reference's CEB builder keeps every column as values plus a null byte per
row, strings as ids of a global string pool (bespoke_ceb/builder_impl.hpp:
97-118, builder_impl.cpp:33-252).  Here a column is an int32 device array
(0 where null; string columns hold the codes of the column's own dictionary,
codes in order of first appearance) and a null byte array when the column
has nulls.  A query's string arguments become per-code byte arrays on the
host (the role of the reference's build_string_id_list over the pool,
bespoke_ceb/query_q1a.cpp:29-42); all row work runs on the GPU.
"""
from __future__ import annotations

import ctypes as C
import re
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import native as N

NULL_WORDS = ("<<NULL>>", "NULL", "null")


def stoi(text: str) -> int | None:
    """std::stoi as the reference calls it: optional leading whitespace and
    sign, then digits (trailing characters ignored); None where stoi throws."""
    m = re.match(r"\s*([+-]?\d+)", text)
    if not m:
        return None
    v = int(m.group(1))
    return v if -2**31 <= v < 2**31 else None


@dataclass
class Column:
    values: object              # torch int32 device tensor
    is_null: object | None      # torch uint8 device tensor, None without nulls
    dictionary: list | None = None   # string columns: code -> value
    max_value: int = -1         # largest non-null value (int columns), -1 without one
    rows: int = 0

    def c(self) -> N.CebCol:
        return N.CebCol(N.ptr(self.values), N.ptr(self.is_null) if self.is_null is not None else None)

    def codes_of(self, values) -> set[int]:
        index = {v: i for i, v in enumerate(self.dictionary or [])}
        return {index[v] for v in values if v in index}


@dataclass
class CebTables:
    tables: dict = field(default_factory=dict)   # table -> {"rows": n, column -> Column}

    def col(self, table: str, name: str) -> Column:
        return self.tables[table][name]

    def rows(self, table: str) -> int:
        return self.tables[table]["rows"]


def _column(arr, torch) -> Column:
    import pyarrow as pa

    arr = arr.combine_chunks() if isinstance(arr, pa.ChunkedArray) else arr
    n = len(arr)
    null = None
    if arr.null_count:
        null = np.asarray(arr.is_null().to_numpy(zero_copy_only=False), dtype=np.uint8)
    if pa.types.is_string(arr.type) or pa.types.is_large_string(arr.type):
        enc = arr.dictionary_encode()
        # codes in order of first appearance (nulls: code 0, flagged in is_null)
        idx = enc.indices.to_numpy(zero_copy_only=False)
        idx = np.where(np.isnan(idx), 0, idx).astype(np.int64) if idx.dtype.kind == "f" else idx.astype(np.int64)
        values = np.asarray(idx, dtype=np.int32)
        dictionary = enc.dictionary.to_pylist()
        mx = -1
    else:
        v = arr.to_numpy(zero_copy_only=False)
        if v.dtype.kind == "f":
            v = np.where(np.isnan(v), 0, v)
        values = np.asarray(v, dtype=np.int64).astype(np.int32)
        dictionary = None
        valid = values[null == 0] if null is not None else values
        mx = int(valid.max()) if len(valid) else -1
    dev = torch.from_numpy(np.ascontiguousarray(values)).cuda()
    ndev = torch.from_numpy(null).cuda() if null is not None else None
    return Column(dev, ndev, dictionary, mx, n)


Q1A_COLUMNS = {
    "title": ("id", "kind_id", "production_year"),
    "movie_info": ("movie_id", "info_type_id", "info"),
    "cast_info": ("movie_id", "person_id", "role_id"),
    "kind_type": ("id", "kind"),
    "role_type": ("id", "role"),
    "name": ("id", "gender"),
    "info_type": ("id",),
}


def load_tables(path: Path, columns: dict = Q1A_COLUMNS) -> CebTables:
    """Reads the named columns of the CEB Parquet files onto the device."""
    import pyarrow.parquet as pq
    import torch

    out = CebTables()
    for table, cols in columns.items():
        t = pq.read_table(Path(path) / f"{table}.parquet", columns=list(cols))
        d = {"rows": t.num_rows}
        for c in cols:
            d[c] = _column(t[c], torch)
        out.tables[table] = d
    return out


def _mask_size(t: CebTables, table: str) -> int:
    """Size of the reference's id masks: row count + 1, grown to hold the
    largest id (query_q1a.cpp:93-115)."""
    return max(t.rows(table) + 1, t.col(table, "id").max_value + 1)


def _code_bytes(col: Column, values) -> np.ndarray:
    out = np.zeros(max(len(col.dictionary or []), 1), np.uint8)
    for c in col.codes_of([v for v in values if v not in NULL_WORDS]):
        out[c] = 1
    return out


def q1a(engine, t: CebTables, id1, id2, info1, info2, kind, role, gender, year1: str, year2: str) -> int:
    """CEB query 1a (run_q1a, bespoke_ceb/query_q1a.cpp:155-655) on the GPU."""
    y1, y2 = stoi(year1), stoi(year2)
    if y1 is None or y2 is None:
        raise ValueError("q1a: YEAR1 / YEAR2 are not integers")
    size_it = _mask_size(t, "info_type")
    tf = np.zeros(max(size_it, 1), np.uint8)
    for bit, ids in ((1, id1), (2, id2)):
        for v in ids:
            if v in NULL_WORDS:
                continue
            i = stoi(v)
            if i is not None and 0 <= i < size_it:
                tf[i] |= bit
    info = t.col("movie_info", "info")
    match = np.zeros(max(len(info.dictionary or []), 1), np.uint8)
    for bit, vals in ((1, info1), (2, info2)):
        for c in info.codes_of([v for v in vals if v not in NULL_WORDS]):
            match[c] |= bit
    ka = _code_bytes(t.col("kind_type", "kind"), kind)
    ra = _code_bytes(t.col("role_type", "role"), role)
    ga = _code_bytes(t.col("name", "gender"), gender)
    tab = N.CebQ1aTables()
    tab.t_id, tab.t_kind_id, tab.t_year = (t.col("title", c).c() for c in ("id", "kind_id", "production_year"))
    tab.n_title = t.rows("title")
    tab.max_title_id = t.col("title", "id").max_value
    tab.mi_movie_id, tab.mi_info_type_id, tab.mi_info = (t.col("movie_info", c).c()
                                                         for c in ("movie_id", "info_type_id", "info"))
    tab.n_movie_info = t.rows("movie_info")
    tab.ci_movie_id, tab.ci_person_id, tab.ci_role_id = (t.col("cast_info", c).c()
                                                         for c in ("movie_id", "person_id", "role_id"))
    tab.n_cast_info = t.rows("cast_info")
    tab.kt_id, tab.kt_kind = t.col("kind_type", "id").c(), t.col("kind_type", "kind").c()
    tab.n_kind_type = t.rows("kind_type")
    tab.rt_id, tab.rt_role = t.col("role_type", "id").c(), t.col("role_type", "role").c()
    tab.n_role_type = t.rows("role_type")
    tab.nm_id, tab.nm_gender = t.col("name", "id").c(), t.col("name", "gender").c()
    tab.n_name = t.rows("name")
    p = N.CebQ1aParams()
    p.year1, p.year2 = y1, y2
    p.info_type_filter, p.info_type_size = tf.ctypes.data, size_it
    p.info_match, p.n_info_codes = match.ctypes.data, len(info.dictionary or [])
    p.kind_allowed, p.n_kind_codes = ka.ctypes.data, len(t.col("kind_type", "kind").dictionary or [])
    p.role_allowed, p.n_role_codes = ra.ctypes.data, len(t.col("role_type", "role").dictionary or [])
    p.gender_allowed, p.n_gender_codes = ga.ctypes.data, len(t.col("name", "gender").dictionary or [])
    p.kind_mask_size = _mask_size(t, "kind_type")
    p.role_mask_size = _mask_size(t, "role_type")
    p.person_mask_size = _mask_size(t, "name")
    out = C.c_int64()
    engine.ctx.call("bo_ceb_q1a", C.byref(tab), C.byref(p), C.byref(out))
    return int(out.value)


# The reference builder's fact-table orders (bespoke_ceb/builder_impl.cpp:432-452).
BUILDER_ORDER = {
    "movie_info": ("movie_id", "info_type_id"),
    "cast_info": ("movie_id", "role_id"),
    "movie_companies": ("movie_id", None),
    "movie_keyword": ("keyword_id", None),
    "person_info": ("info_type_id", None),
    "name": ("id", None),
    "title": ("id", None),
}


def sort_table(engine, t: CebTables, table: str, primary: str, secondary: str | None = None) -> None:
    """Reorders every loaded column of `table` on the device by (primary,
    secondary) -- the builder's order for that table -- keeping ties in their
    input order."""
    import torch

    d = t.tables[table]
    n = d["rows"]
    if n == 0:
        return
    perm = torch.empty(n, dtype=torch.int32, device="cuda")
    sec = d[secondary].values if secondary else None
    engine.ctx.call("bo_ceb_sort_rows", C.c_void_p(N.ptr(d[primary].values)), C.c_void_p(N.ptr(sec)), n,
                    C.c_void_p(perm.data_ptr()))
    for name, col in list(d.items()):
        if name == "rows":
            continue
        v = torch.empty_like(col.values)
        engine.ctx.call("bo_ceb_gather_i32", C.c_void_p(col.values.data_ptr()), C.c_void_p(perm.data_ptr()), n,
                        C.c_void_p(v.data_ptr()))
        nl = None
        if col.is_null is not None:
            nl = torch.empty_like(col.is_null)
            engine.ctx.call("bo_ceb_gather_u8", C.c_void_p(col.is_null.data_ptr()), C.c_void_p(perm.data_ptr()), n,
                            C.c_void_p(nl.data_ptr()))
        d[name] = Column(v, nl, col.dictionary, col.max_value, col.rows)
    engine.synchronize()


def builder_order(engine, t: CebTables) -> None:
    """Applies the builder's order to every loaded table that has one."""
    for table, (p, s) in BUILDER_ORDER.items():
        if table in t.tables and p in t.tables[table] and (s is None or s in t.tables[table]):
            sort_table(engine, t, table, p, s)
