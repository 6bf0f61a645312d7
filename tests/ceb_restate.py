"""A plain-Python restatement of CEB query 1a (run_q1a,
bespoke_ceb/query_q1a.cpp:155-655) over the Parquet files, for the tests:
the reference's id masks, null skips, dense per-movie counts and the
factorised sum over the qualifying title rows."""
from __future__ import annotations

import re
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


def q10a(path, ids, infos, name, kinds, roles, pool) -> list:
    """run_q10a (bespoke_ceb/query_q10a.cpp:334-1130) restated: rows
    (name, info, min year, max year) -- years None without one -- sorted."""
    from bespokeolap_artifacts_b200.ceb import ascii_lower, ilike_pattern, string_filter

    type_ids = {i for i in (stoi(v) for v in ids if v not in NULL_WORDS) if i is not None}
    kf, rf, inf = string_filter(pool, kinds), string_filter(pool, roles), string_filter(pool, infos)
    if not type_ids or not kf or not rf or not inf:
        return []
    (it_ids,), n_it = _cols(path, "info_type", ("id",))
    tmask = {i for i in type_ids if 0 <= i < n_it + 1}
    (kid, kk), n_k = _cols(path, "kind_type", ("id", "kind"))
    kinds_ok = {i for i, v in zip(kid, kk) if i is not None and v is not None and 0 <= i < n_k + 1 and v in kf}
    (rid, rr), n_r = _cols(path, "role_type", ("id", "role"))
    roles_ok = {i for i, v in zip(rid, rr) if i is not None and v is not None and 0 <= i < n_r + 1 and v in rf}
    if not tmask or not kinds_ok or not roles_ok:
        return []
    (tid, tkind, tyear), n_t = _cols(path, "title", ("id", "kind_id", "production_year"))
    present, year = set(), {}
    for i, k, y in zip(tid, tkind, tyear):
        if i is None or k is None or k not in kinds_ok or not 0 <= i < n_t + 1:
            continue
        present.add(i)
        year[i] = y
    (mm, mt, mi), _ = _cols(path, "movie_info", ("movie_id", "info_type_id", "info"))
    infos_of = {}
    for m, ty, v in zip(mm, mt, mi):
        if ty is None or v is None or ty not in tmask or v not in inf or m is None or m not in present:
            continue
        infos_of.setdefault(m, []).append(v)
    (nid, nname), n_n = _cols(path, "name", ("id", "name"))
    (cm, cp, cr), _ = _cols(path, "cast_info", ("movie_id", "person_id", "role_id"))
    pairs = [(m, p) for m, p, r in zip(cm, cp, cr)
             if m is not None and p is not None and r is not None and m in infos_of and r in roles_ok
             and 0 <= p < n_n + 1]
    cand = {p for _, p in pairs}
    ptype, pat = ilike_pattern(name)

    def like(s: str) -> bool:
        s = ascii_lower(s)
        if ptype == 0:
            return True
        if ptype == 1:
            return s == pat
        if ptype == 2:
            return s.startswith(pat)
        if ptype == 3:
            return s.endswith(pat)
        if ptype == 4:
            return pat in s
        return re.fullmatch("".join(".*" if c == "%" else "." if c == "_" else re.escape(c) for c in pat), s,
                            re.S) is not None

    pname = {}
    for i, nm in zip(nid, nname):
        if i is None or nm is None or i not in cand or not like(nm):
            continue
        pname[i] = nm
    agg = {}
    for m, p in pairs:
        if p not in pname:
            continue
        y = year.get(m)
        for v in infos_of[m]:
            key = (pname[p], v)
            lo, hi = agg.get(key, (None, None))
            if y is not None:
                lo = y if lo is None else min(lo, y)
                hi = y if hi is None else max(hi, y)
            agg[key] = (lo, hi)
    return sorted((n, v, lo, hi) for (n, v), (lo, hi) in agg.items())


def _like(ptype: int, pat: str, s: str) -> bool:
    from bespokeolap_artifacts_b200.ceb import ascii_lower

    s = ascii_lower(s)
    if ptype == 0:
        return True
    if ptype == 1:
        return s == pat
    if ptype == 2:
        return s.startswith(pat)
    if ptype == 3:
        return s.endswith(pat)
    if ptype == 4:
        return pat in s
    return re.fullmatch("".join(".*" if c == "%" else "." if c == "_" else re.escape(c) for c in pat), s,
                        re.S) is not None


def q3b(path, title, pcode, company, kinds, roles) -> list:
    """run_q3b (bespoke_ceb/query_q3b.cpp:728-1420) restated: per movie the
    movie_companies counts of companies whose name matches, the
    movie_keyword count, the title (allowed kind, matching title), the
    cast_info counts of persons of an allowed role whose pcode matches;
    count = keywords x cast x companies per (title, name, company), ordered
    by count desc, title, name, company."""
    from bespokeolap_artifacts_b200.ceb import ilike_pattern, string_filter

    tp, pp, cp = ilike_pattern(title), ilike_pattern(pcode), ilike_pattern(company)
    (kid, kk), n_k = _cols(path, "kind_type", ("id", "kind"))
    kf = string_filter({v for v in kk if v is not None}, kinds)
    kinds_ok = {i for i, v in zip(kid, kk) if i is not None and v is not None and i >= 0 and v in kf}
    (rid, rr), n_r = _cols(path, "role_type", ("id", "role"))
    rf = string_filter({v for v in rr if v is not None}, roles)
    roles_ok = {i for i, v in zip(rid, rr) if i is not None and v is not None and i >= 0 and v in rf}
    if not kinds_ok or not roles_ok:
        return []
    (cid, cname), _ = _cols(path, "company_name", ("id", "name"))
    comp = {}
    for i, nm in zip(cid, cname):
        if i is not None and nm is not None and i >= 0 and _like(*cp, nm):
            comp[i] = nm
    if not comp:
        return []
    (mm, mc, mt), _ = _cols(path, "movie_companies", ("movie_id", "company_id", "company_type_id"))
    mc_by = {}
    for m, c, ty in zip(mm, mc, mt):
        if m is None or c is None or ty is None or c not in comp:
            continue
        d = mc_by.setdefault(m, {})
        d[c] = d.get(c, 0) + 1
    (km, kw), _ = _cols(path, "movie_keyword", ("movie_id", "keyword_id"))
    mk = {}
    for m, k in zip(km, kw):
        if m is None or k is None or m not in mc_by:
            continue
        mk[m] = mk.get(m, 0) + 1
    cand = {m for m in mc_by if mk.get(m)}
    (tid, ttitle, tkind), _ = _cols(path, "title", ("id", "title", "kind_id"))
    titles = {}
    for i, tt, k in zip(tid, ttitle, tkind):
        if i is None or i not in cand or i in titles or tt is None or k is None or k not in kinds_ok:
            continue
        if _like(*tp, tt):
            titles[i] = tt
    (cm, cpers, crole), _ = _cols(path, "cast_info", ("movie_id", "person_id", "role_id"))
    ci_by = {}
    for m, p, r in zip(cm, cpers, crole):
        if m is None or p is None or r is None or m not in titles or r not in roles_ok:
            continue
        d = ci_by.setdefault(m, {})
        d[p] = d.get(p, 0) + 1
    persons = {p for d in ci_by.values() for p in d if p >= 0}
    (nid, nname, npc), _ = _cols(path, "name", ("id", "name", "name_pcode_nf"))
    pname = {}
    for i, nm, pc in zip(nid, nname, npc):
        if i is None or i not in persons or i in pname or nm is None or pc is None:
            continue
        if _like(*pp, pc):
            pname[i] = nm
    out = {}
    for m, d in ci_by.items():
        for p, ci in d.items():
            if p not in pname:
                continue
            for c, n in mc_by[m].items():
                key = (titles[m], pname[p], comp[c])
                out[key] = out.get(key, 0) + mk[m] * ci * n
    return sorted(((t, n, c, v) for (t, n, c), v in out.items()), key=lambda r: (-r[3], r[0], r[1], r[2]))
