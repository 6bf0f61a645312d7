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
from dataclasses import dataclass, field, replace
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
    dict_bytes: object = None   # string columns: the dictionary's bytes and
    dict_offsets: object = None  # n + 1 uint32 offsets, on the device
    dict_rank: object = None    # string columns: each code's position in string order (device)

    def dict_c(self) -> N.CebDict:
        return N.CebDict(N.ptr(self.dict_bytes), N.ptr(self.dict_offsets), N.ptr(self.dict_rank),
                         len(self.dictionary or []))

    def c(self) -> N.CebCol:
        return N.CebCol(N.ptr(self.values), N.ptr(self.is_null) if self.is_null is not None else None)

    def codes_of(self, values) -> set[int]:
        index = {v: i for i, v in enumerate(self.dictionary or [])}
        return {index[v] for v in values if v in index}


@dataclass
class CebTables:
    tables: dict = field(default_factory=dict)   # table -> {"rows": n, column -> Column}
    pool: set = field(default_factory=set)       # every string of the database (the reference's pool)

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
        raw = [v.encode() for v in dictionary]
        offs = np.zeros(len(raw) + 1, np.uint32)
        offs[1:] = np.cumsum([len(b) for b in raw], dtype=np.int64).astype(np.uint32) if raw else []
        blob = np.frombuffer(b"".join(raw) or b"\0", dtype=np.uint8)
        rank = np.empty(max(len(dictionary), 1), np.int32)
        rank[np.array(sorted(range(len(dictionary)), key=lambda i: raw[i]), dtype=np.int64)] = np.arange(
            len(dictionary), dtype=np.int32)
        dict_dev = (torch.from_numpy(blob.copy()).cuda(), torch.from_numpy(offs.view(np.int32).copy()).cuda(),
                    torch.from_numpy(rank).cuda())
    else:
        v = arr.to_numpy(zero_copy_only=False)
        if v.dtype.kind == "f":
            v = np.where(np.isnan(v), 0, v)
        values = np.asarray(v, dtype=np.int64).astype(np.int32)
        dictionary = None
        dict_dev = (None, None, None)
        valid = values[null == 0] if null is not None else values
        mx = int(valid.max()) if len(valid) else -1
    dev = torch.from_numpy(np.ascontiguousarray(values)).cuda()
    ndev = torch.from_numpy(null).cuda() if null is not None else None
    return Column(dev, ndev, dictionary, mx, n, *dict_dev)


Q1A_COLUMNS = {
    "title": ("id", "kind_id", "production_year"),
    "movie_info": ("movie_id", "info_type_id", "info"),
    "cast_info": ("movie_id", "person_id", "role_id"),
    "kind_type": ("id", "kind"),
    "role_type": ("id", "role"),
    "name": ("id", "gender"),
    "info_type": ("id",),
}


Q10A_COLUMNS = {
    "title": ("id", "kind_id", "production_year"),
    "movie_info": ("movie_id", "info_type_id", "info"),
    "cast_info": ("movie_id", "person_id", "role_id"),
    "kind_type": ("id", "kind"),
    "role_type": ("id", "role"),
    "name": ("id", "name"),
    "info_type": ("id",),
}


Q3B_COLUMNS = {
    "kind_type": ("id", "kind"),
    "role_type": ("id", "role"),
    "company_name": ("id", "name"),
    "movie_companies": ("movie_id", "company_id", "company_type_id"),
    "movie_keyword": ("movie_id", "keyword_id"),
    "title": ("id", "title", "kind_id"),
    "cast_info": ("movie_id", "person_id", "role_id"),
    "name": ("id", "name", "name_pcode_nf"),
}


def string_pool(path: Path) -> set:
    """Every string value of every table (the reference interns all of them
    into one pool, bespoke_ceb/builder_impl.cpp:408-422)."""
    import pyarrow as pa
    import pyarrow.parquet as pq

    pool = set()
    for f in sorted(Path(path).glob("*.parquet")):
        t = pq.read_table(f)
        for c in t.column_names:
            if pa.types.is_string(t[c].type) or pa.types.is_large_string(t[c].type):
                pool.update(v for v in t[c].unique().to_pylist() if v is not None)
    return pool


def load_tables(path: Path, columns: dict = Q1A_COLUMNS) -> CebTables:
    """Reads the named columns of the CEB Parquet files onto the device."""
    import pyarrow.parquet as pq
    import torch

    out = CebTables(pool=string_pool(path))
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
        d[name] = replace(col, values=v, is_null=nl)  # the device dictionary stays with the codes
    engine.synchronize()


def builder_order(engine, t: CebTables) -> None:
    """Applies the builder's order to every loaded table that has one."""
    for table, (p, s) in BUILDER_ORDER.items():
        if table in t.tables and p in t.tables[table] and (s is None or s in t.tables[table]):
            sort_table(engine, t, table, p, s)


# ------------------------------------------------------------------ 10a ----
def string_filter(pool: set, values) -> set:
    """build_string_filter_for_column (bespoke_ceb/query_q10a.cpp:248-282):
    IN-list values were split at commas by the request parser, so runs of
    consecutive values are re-joined with ", " or "," and the longest run
    that names a string of the database is taken."""
    out, i = set(), 0
    while i < len(values):
        if values[i] in NULL_WORDS:
            i += 1
            continue
        sp = nsp = values[i]
        found, found_idx = None, i
        for j in range(i, len(values)):
            if j != i:
                if values[j] in NULL_WORDS:
                    break
                sp += ", " + values[j]
                nsp += "," + values[j]
            if sp in pool:
                found, found_idx = sp, j
            if nsp in pool:
                found, found_idx = nsp, j
        if found is not None:
            out.add(found)
            i = found_idx + 1
        else:
            i += 1
    return out


def ascii_lower(s: str) -> str:
    return "".join(chr(ord(c) + 32) if "A" <= c <= "Z" else c for c in s)


def ilike_pattern(raw: str) -> tuple[int, str]:
    """build_ilike_pattern (bespoke_ceb/query_q10a.cpp:172-214): the pattern
    kind (0 all, 1 exact, 2 prefix, 3 suffix, 4 contains, 5 general) and its
    lower-cased token or pattern."""
    p = raw[1:-1] if len(raw) >= 2 and raw[0] == "'" and raw[-1] == "'" else raw
    p = ascii_lower(p)
    if p == "%":
        return 0, ""
    if "_" not in p:
        first = p.find("%")
        if first < 0:
            return 1, p
        last = p.rfind("%")
        if first == 0 and last == len(p) - 1 and p.find("%", 1) == last:
            return 4, p[1:-1] if len(p) > 2 else ""
        if first == 0 and p.find("%", 1) < 0:
            return 3, p[1:]
        if last == len(p) - 1 and p.find("%") == last:
            return 2, p[:-1]
    return 5, p


def q10a(engine, t: CebTables, ids, infos, name, kinds, roles, max_rows: int = 1 << 16, raw: bool = False):
    """CEB query 10a (run_q10a, bespoke_ceb/query_q10a.cpp:334-1130) on the
    GPU: rows (name, info, has_year, min_year, max_year), in no particular
    order (the reference's are in its aggregation order).  raw=True returns
    the row count instead (the rows stay as codes: no strings are built)."""
    max_rows = max(max_rows, getattr(q10a, "room", 0))
    type_ids = {i for i in (stoi(v) for v in ids if v not in NULL_WORDS) if i is not None}
    if not type_ids:
        return []
    kf, rf, inf = string_filter(t.pool, kinds), string_filter(t.pool, roles), string_filter(t.pool, infos)
    if not kf or not rf or not inf:
        return []
    size_it = t.rows("info_type") + 1
    tmask = np.zeros(size_it, np.uint8)
    for i in type_ids:
        if 0 <= i < size_it:
            tmask[i] = 1
    if not tmask.any():
        return []
    info = t.col("movie_info", "info")
    dense_vals = sorted(inf)
    dense_of = {v: k for k, v in enumerate(dense_vals)}
    info_dense = np.full(max(len(info.dictionary or []), 1), -1, np.int32)
    for c, v in enumerate(info.dictionary or []):
        if v in dense_of:
            info_dense[c] = dense_of[v]
    ka = _code_bytes(t.col("kind_type", "kind"), kf)
    ra = _code_bytes(t.col("role_type", "role"), rf)
    ptype, pat = ilike_pattern(name)
    pat_b = pat.encode()
    pat_buf = np.frombuffer(pat_b or b"\0", np.uint8).copy()
    nm = t.col("name", "name")
    tab = N.CebQ10aTables()
    tab.t_id, tab.t_kind_id, tab.t_year = (t.col("title", c).c() for c in ("id", "kind_id", "production_year"))
    tab.n_title = t.rows("title")
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
    tab.nm_id, tab.nm_name = t.col("name", "id").c(), nm.c()
    tab.n_name = t.rows("name")
    tab.name_dict, tab.name_dict_offsets = N.ptr(nm.dict_bytes), N.ptr(nm.dict_offsets)
    tab.n_name_codes = len(nm.dictionary or [])
    p = N.CebQ10aParams()
    p.info_type_mask, p.info_type_size = tmask.ctypes.data, size_it
    p.info_dense, p.n_info_codes, p.n_info_dense = info_dense.ctypes.data, len(info.dictionary or []), len(dense_vals)
    p.kind_allowed, p.n_kind_codes = ka.ctypes.data, len(t.col("kind_type", "kind").dictionary or [])
    p.role_allowed, p.n_role_codes = ra.ctypes.data, len(t.col("role_type", "role").dictionary or [])
    p.pattern_type, p.pattern, p.pattern_len = ptype, pat_buf.ctypes.data, len(pat_b)
    while True:
        rows = (N.CebQ10aRow * max(max_rows, 1))()
        n, dense = C.c_int64(), C.c_int32()
        rc = N.lib().bo_ceb_q10a(engine.ctx.handle, C.byref(tab), C.byref(p), rows, max_rows, C.byref(n),
                                 C.byref(dense))
        if rc == N.BO_ERR_OVERFLOW and n.value > max_rows:
            max_rows = int(n.value)  # more groups than rows offered: run again with room for all
            continue
        engine.ctx.check(rc, "bo_ceb_q10a")
        break
    q10a.room = max_rows
    if raw:
        return int(n.value)
    out = []
    for r in rows[:n.value]:
        out.append((nm.dictionary[r.name_code], dense_vals[r.info_dense], bool(r.has_year),
                    r.min_year if r.has_year else None, r.max_year if r.has_year else None))
    q10a.last_dense = bool(dense.value)
    return out


# ------------------------------------------------------------------- 3b ----
def q3b(engine, t: CebTables, title: str, pcode: str, company: str, kinds, roles, max_rows: int = 1 << 16,
        raw: bool = False):
    """CEB query 3b (run_q3b, bespoke_ceb/query_q3b.cpp:728-1420) on the GPU:
    rows (title, name, company, count) in the reference's order (count desc,
    then the three strings).  raw=True returns the row count instead."""
    max_rows = max(max_rows, getattr(q3b, "room", 0))
    kt, rt = t.col("kind_type", "kind"), t.col("role_type", "role")
    # the IN lists against the column's own strings (query_q3b.cpp:208-254)
    kf = string_filter(set(kt.dictionary or []), kinds)
    rf = string_filter(set(rt.dictionary or []), roles)
    ka, ra = _code_bytes(kt, kf), _code_bytes(rt, rf)
    pats = [ilike_pattern(x) for x in (title, pcode, company)]
    bufs = [np.frombuffer(pt.encode() or b"\0", np.uint8).copy() for _, pt in pats]
    tab = N.CebQ3bTables()
    tab.kt_id, tab.kt_kind, tab.n_kind_type = t.col("kind_type", "id").c(), kt.c(), t.rows("kind_type")
    tab.rt_id, tab.rt_role, tab.n_role_type = t.col("role_type", "id").c(), rt.c(), t.rows("role_type")
    cn = t.col("company_name", "name")
    tab.cn_id, tab.cn_name, tab.n_company_name = t.col("company_name", "id").c(), cn.c(), t.rows("company_name")
    tab.mc_movie_id, tab.mc_company_id, tab.mc_company_type_id = (
        t.col("movie_companies", c).c() for c in ("movie_id", "company_id", "company_type_id"))
    tab.n_movie_companies = t.rows("movie_companies")
    tab.mk_movie_id, tab.mk_keyword_id = (t.col("movie_keyword", c).c() for c in ("movie_id", "keyword_id"))
    tab.n_movie_keyword = t.rows("movie_keyword")
    tt = t.col("title", "title")
    tab.t_id, tab.t_title, tab.t_kind_id = t.col("title", "id").c(), tt.c(), t.col("title", "kind_id").c()
    tab.n_title = t.rows("title")
    tab.ci_movie_id, tab.ci_person_id, tab.ci_role_id = (t.col("cast_info", c).c()
                                                         for c in ("movie_id", "person_id", "role_id"))
    tab.n_cast_info = t.rows("cast_info")
    nm, pc = t.col("name", "name"), t.col("name", "name_pcode_nf")
    tab.nm_id, tab.nm_name, tab.nm_pcode, tab.n_name = t.col("name", "id").c(), nm.c(), pc.c(), t.rows("name")
    tab.title_dict, tab.name_dict, tab.company_dict, tab.pcode_dict = tt.dict_c(), nm.dict_c(), cn.dict_c(), pc.dict_c()
    tab.movie_bound = max(t.col("movie_companies", "movie_id").max_value, -1) + 1
    tab.person_bound = max(t.col("cast_info", "person_id").max_value, -1) + 1
    p = N.CebQ3bParams()
    p.kind_allowed, p.role_allowed = ka.ctypes.data, ra.ctypes.data
    p.n_kind_codes, p.n_role_codes = len(kt.dictionary or []), len(rt.dictionary or [])
    p.kind_mask_size, p.role_mask_size = _mask_size(t, "kind_type"), _mask_size(t, "role_type")
    p.company_map_size = _mask_size(t, "company_name")
    (p.title_type, _), (p.pcode_type, _), (p.company_type, _) = pats
    p.title_pat, p.pcode_pat, p.company_pat = (b.ctypes.data for b in bufs)
    p.title_len, p.pcode_len, p.company_len = (len(pt.encode()) for _, pt in pats)
    while True:
        rows = (N.CebQ3bRow * max(max_rows, 1))()
        n = C.c_int64()
        rc = N.lib().bo_ceb_q3b(engine.ctx.handle, C.byref(tab), C.byref(p), rows, max_rows, C.byref(n))
        if rc == N.BO_ERR_OVERFLOW and n.value > max_rows:
            max_rows = int(n.value)  # more groups than rows offered: run again with room for all
            continue
        engine.ctx.check(rc, "bo_ceb_q3b")
        break
    q3b.room = max_rows
    if raw:
        return int(n.value)
    return [(tt.dictionary[r.title_code], nm.dictionary[r.name_code], cn.dictionary[r.company_code], int(r.count))
            for r in rows[:n.value]]
