"""ORACLE -- test infrastructure, not part of the product.

Python access to the CPU checker:
  * ``liboracle.so``  -- the plain-C restatement of the reference pipelines
    (``bo_oracle.c``);
  * ``_ref/libref_tpch.so`` / ``_ref/libref_tpch_trace.so`` -- the reference's own
    TPC-H pipelines compiled unchanged (``ref_harness.cpp``).

Only tests, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline / reference
legs import this module, and only to check or to time the CPU path.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_P = C.c_void_p


def _p(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


class OI128(C.Structure):
    _fields_ = [("lo", C.c_uint64), ("hi", C.c_int64)]

    def value(self) -> int:
        return (self.hi << 64) | self.lo


class OQ1Agg(C.Structure):
    _fields_ = [
        ("count", C.c_int64), ("sum_qty", C.c_int64), ("sum_base_price", C.c_int64), ("sum_disc", C.c_int64),
        ("sum_disc_price", C.c_int64), ("sum_disc_price_exact", C.c_int64),
        ("sum_charge", OI128), ("sum_charge_exact", OI128),
    ]

    def as_dict(self) -> dict:
        d = {f: getattr(self, f) for f, _ in self._fields_[:6]}
        d["sum_charge"] = self.sum_charge.value()
        d["sum_charge_exact"] = self.sum_charge_exact.value()
        return d


_olib = None


def olib() -> C.CDLL:
    global _olib
    if _olib is None:
        path = HERE / "liboracle.so"
        if not path.exists():
            raise RuntimeError(f"{path} missing: run `python oracle/build_oracle.py`")
        _olib = C.CDLL(str(path))
        _olib.oracle_q1_fact.argtypes = [_P] * 7 + [C.c_int64, C.c_int32, C.c_int32, C.c_int32, _P]
        _olib.oracle_q1_lineitem.argtypes = [_P] * 7 + [C.c_int64, C.c_int16, C.c_int32, _P]
        _olib.oracle_q1_finalize.argtypes = [_P, _P]
        _olib.oracle_q1_finalize.restype = None
        _olib.oracle_q6_lineitem.argtypes = [_P] * 4 + [C.c_int64, C.c_int16, C.c_int16, C.c_int32, C.c_int32,
                                                        C.c_int32, _P, _P]
        _olib.oracle_join_agg.argtypes = [_P, _P, _P, C.c_int64, C.c_int32, C.c_int32, _P, _P, _P, C.c_int64,
                                          _P, _P, _P, _P]
        _olib.oracle_groupby_topk.restype = C.c_int64
        _olib.oracle_groupby_topk.argtypes = [_P, C.c_int64, _P, _P, C.c_int64, _P, _P, C.c_int64, _P, C.c_int32,
                                              C.c_int32, C.c_int32, C.c_int32, _P, _P, _P, _P]
        _olib.oracle_distinct_groups.restype = C.c_int64
        _olib.oracle_distinct_groups.argtypes = [_P, C.c_int64, _P, _P, C.c_int64, _P, _P, C.c_int64, _P,
                                                 C.c_int32, C.c_int32, C.c_int32]
        _olib.oracle_radix_sort_pairs.argtypes = [_P, _P, C.c_int64]
    return _olib


# ------------------------------------------------------------------- Q1 -----
def q1_fact(t, cutoff: int) -> tuple[list[dict], int]:
    ng = t.n_flag_a * t.n_flag_b
    out = (OQ1Agg * ng)()
    cols = [np.ascontiguousarray(c) for c in t.columns()]
    rc = olib().oracle_q1_fact(*[_p(c) for c in cols], t.n_rows, cutoff, t.n_flag_a, t.n_flag_b, out)
    return [out[g].as_dict() for g in range(ng)], rc


def q1_lineitem(cols: dict, cutoff: int, n_groups: int) -> tuple[list[dict], int]:
    out = (OQ1Agg * n_groups)()
    names = ["shipdate", "returnflag_linestatus", "extendedprice", "discounted_price", "discount", "tax", "quantity"]
    arrs = [np.ascontiguousarray(cols[k]) for k in names]
    rc = olib().oracle_q1_lineitem(*[_p(a) for a in arrs], len(arrs[0]), cutoff, n_groups, out)
    return [out[g].as_dict() for g in range(n_groups)], rc


def q1_finalize(agg: dict) -> list[float]:
    """run_q1's integer-to-double finalisation (query_q1.cpp:245-257) in C."""
    a = OQ1Agg()
    for k in ("count", "sum_qty", "sum_base_price", "sum_disc", "sum_disc_price", "sum_disc_price_exact"):
        setattr(a, k, agg[k])
    ch = agg["sum_charge"]
    a.sum_charge.lo = ch & ((1 << 64) - 1)
    a.sum_charge.hi = ch >> 64
    out = (C.c_double * 7)()
    olib().oracle_q1_finalize(C.byref(a), out)
    return list(out)


def q6_lineitem(cols: dict, start: int, end: int, dmin: int, dmax: int, qlimit: int) -> tuple[int, int]:
    arrs = [np.ascontiguousarray(cols[k]) for k in ("shipdate", "extendedprice", "discount", "quantity")]
    rev = C.c_int64()
    cnt = C.c_int64()
    olib().oracle_q6_lineitem(*[_p(a) for a in arrs], len(arrs[0]), start, end, dmin, dmax, qlimit,
                              C.byref(rev), C.byref(cnt))
    return rev.value, cnt.value


# ----------------------------------------------------------------- join -----
def join_agg(j) -> dict:
    bc, mc = C.c_int64(), C.c_int64()
    se, st = OI128(), OI128()
    olib().oracle_join_agg(_p(j.b_key), _p(j.b_date), _p(j.b_seg), j.n_build, j.date_lt, j.seg_eq,
                           _p(j.p_fk), _p(j.p_price), _p(j.p_disc), j.n_probe,
                           C.byref(bc), C.byref(mc), C.byref(se), C.byref(st))
    return dict(build_count=bc.value, match_count=mc.value, sum_exact=se.value(), sum_trunc=st.value())


# -------------------------------------------------------------- group-by ----
def groupby_topk(g, k: int | None = None) -> dict:
    k = g.k if k is None else k
    ok = np.zeros(max(k, 1), np.int32)
    oc = np.zeros(max(k, 1), np.int64)
    oy = np.zeros(max(k, 1), np.int32)
    joined = C.c_int64()
    ng = olib().oracle_groupby_topk(_p(g.a_ids), len(g.a_ids), _p(g.b_a), _p(g.b_c), len(g.b_a),
                                    _p(g.c_cat), _p(g.c_year), len(g.c_cat), _p(g.cat_set), len(g.cat_set),
                                    g.year_lo, g.year_hi, k, _p(ok), _p(oc), _p(oy), C.byref(joined))
    if ng < 0:
        raise RuntimeError(f"oracle_groupby_topk failed: {ng}")
    n = min(k, ng)
    return dict(n_groups=ng, joined_rows=joined.value, keys=ok[:n].tolist(), counts=oc[:n].tolist(),
                min_years=oy[:n].tolist())


def radix_sort_pairs(keys: np.ndarray, vals: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    k = np.ascontiguousarray(keys, dtype=np.uint64).copy()
    v = np.ascontiguousarray(vals, dtype=np.uint32).copy()
    olib().oracle_radix_sort_pairs(_p(k), _p(v), len(k))
    return k, v


# ---------------------------------------------- compiled reference pipelines --
class RefTpchInput(C.Structure):
    _fields_ = [
        ("n_lineitem", C.c_int64), ("l_orderkey", _P), ("l_shipdate", _P), ("l_quantity", _P),
        ("l_extendedprice", _P), ("l_discount", _P), ("l_tax", _P), ("l_returnflag", _P), ("l_linestatus", _P),
        ("n_orders", C.c_int64), ("o_orderkey", _P), ("o_custkey", _P), ("o_orderdate", _P),
        ("n_customer", C.c_int64), ("c_custkey", _P), ("c_mktsegment", _P),
    ]


class RefQ1Row(C.Structure):
    _fields_ = [("returnflag", C.c_char * 8), ("linestatus", C.c_char * 8)] + [
        (f, C.c_double) for f in ("sum_qty", "sum_base_price", "sum_disc_price", "sum_charge", "avg_qty",
                                  "avg_price", "avg_disc")] + [("count_order", C.c_int64)]


class RefLineitemView(C.Structure):
    _fields_ = [
        ("shipdate", _P), ("returnflag_linestatus", _P), ("extendedprice", _P), ("discounted_price", _P),
        ("discount", _P), ("tax", _P), ("quantity", _P), ("n_rows", C.c_int64), ("returnflag_count", C.c_int32),
        ("linestatus_count", C.c_int32), ("base_date_days", C.c_int32), ("orderkey_sorted", C.c_int32),
    ]


_ref_libs: dict[bool, C.CDLL] = {}


def ref_available(trace: bool = False) -> bool:
    return (HERE / "_ref" / ("libref_tpch_trace.so" if trace else "libref_tpch.so")).exists()


def ref_lib(trace: bool = False) -> C.CDLL:
    if trace not in _ref_libs:
        path = HERE / "_ref" / ("libref_tpch_trace.so" if trace else "libref_tpch.so")
        if not path.exists():
            raise RuntimeError(f"{path} missing: build it with `python oracle/build_oracle.py` where the "
                               "reference sources are present")
        l = C.CDLL(str(path))
        l.ref_tpch_build.restype = _P
        l.ref_tpch_build.argtypes = [C.POINTER(RefTpchInput), C.POINTER(C.c_double), C.c_char_p, C.c_int]
        l.ref_tpch_free.argtypes = [_P]
        l.ref_tpch_free.restype = None
        l.ref_lineitem.argtypes = [_P, C.POINTER(RefLineitemView), C.c_char_p, C.c_char_p]
        l.ref_q1.argtypes = [_P, C.c_int32, C.POINTER(RefQ1Row), C.c_int, C.POINTER(C.c_double)]
        l.ref_q3.restype = C.c_int64
        l.ref_q3.argtypes = [_P, C.c_int32, C.c_char_p, C.POINTER(C.c_int64), _P, _P, C.c_int64,
                             C.POINTER(C.c_double)]
        l.ref_q18.restype = C.c_int64
        l.ref_q18.argtypes = [_P, C.c_char_p, _P, _P, C.c_int64, C.POINTER(C.c_double)]
        l.ref_q6.argtypes = [_P, C.c_char_p, C.c_char_p, C.c_char_p, C.POINTER(C.c_int64), C.POINTER(C.c_double)]
        l.ref_parallel.restype = C.c_double
        l.ref_parallel.argtypes = [C.POINTER(_P), C.c_int, C.c_int, C.c_int32, C.c_int32, C.c_char_p,
                                   C.POINTER(C.c_int64)]
        l.ref_trace_begin.argtypes = []
        l.ref_trace_begin.restype = None
        l.ref_trace_end.argtypes = [C.c_char_p, C.c_int]
        _ref_libs[trace] = l
    return _ref_libs[trace]


class RefDatabase:
    """A reference ``Database`` built by the reference's own build()."""

    def __init__(self, tables: dict, trace: bool = False):
        self.lib = ref_lib(trace)
        self.trace = trace
        self._keep = {}
        inp = RefTpchInput()
        for name, _ in RefTpchInput._fields_:
            v = tables.get(name)
            if name.startswith("n_"):
                setattr(inp, name, int(v))
            elif v is not None:
                arr = np.ascontiguousarray(v)
                self._keep[name] = arr
                setattr(inp, name, arr.ctypes.data)
        err = C.create_string_buffer(512)
        ms = C.c_double()
        h = self.lib.ref_tpch_build(C.byref(inp), C.byref(ms), err, 512)
        if not h:
            raise RuntimeError(f"reference build() failed: {err.value.decode()}")
        self.handle = h
        self.build_ms = ms.value
        self._keep.clear()

    def close(self):
        if self.handle:
            self.lib.ref_tpch_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def lineitem(self) -> dict:
        """The storage-plan lineitem columns the reference builder derived
        (views; valid while this database lives)."""
        v = RefLineitemView()
        rf = C.create_string_buffer(16)
        ls = C.create_string_buffer(16)
        self.lib.ref_lineitem(self.handle, C.byref(v), rf, ls)
        n = v.n_rows

        def view(p, dt):
            if n == 0:
                return np.zeros(0, dt)
            return np.ctypeslib.as_array(C.cast(p, C.POINTER(np.ctypeslib.as_ctypes_type(dt))), shape=(n,))

        return dict(
            shipdate=view(v.shipdate, np.int16), returnflag_linestatus=view(v.returnflag_linestatus, np.uint8),
            extendedprice=view(v.extendedprice, np.int32), discounted_price=view(v.discounted_price, np.int32),
            discount=view(v.discount, np.uint8), tax=view(v.tax, np.uint8), quantity=view(v.quantity, np.int16),
            n_rows=n, returnflag_count=v.returnflag_count, linestatus_count=v.linestatus_count,
            returnflag_dict=rf.value.decode(), linestatus_dict=ls.value.decode(),
            base_date_days=v.base_date_days, orderkey_sorted=bool(v.orderkey_sorted),
        )

    def q1(self, delta_days: int = 90) -> tuple[list[dict], float]:
        rows = (RefQ1Row * 16)()
        ms = C.c_double()
        n = self.lib.ref_q1(self.handle, delta_days, rows, 16, C.byref(ms))
        out = []
        for r in rows[:n]:
            d = {f: getattr(r, f) for f, _ in RefQ1Row._fields_}
            d["returnflag"] = r.returnflag.decode()
            d["linestatus"] = r.linestatus.decode()
            out.append(d)
        return out, ms.value

    def q3(self, segment: int, date: str, want_rows: bool = False) -> dict:
        s = C.c_int64()
        ms = C.c_double()
        if self.trace:
            self.lib.ref_trace_begin()
        n = self.lib.ref_q3(self.handle, segment, date.encode(), C.byref(s), None, None, 0, C.byref(ms))
        out = dict(n_rows=n, revenue_sum=s.value, ms=ms.value)
        if self.trace:
            buf = C.create_string_buffer(1 << 16)
            self.lib.ref_trace_end(buf, 1 << 16)
            out["trace"] = parse_trace(buf.value.decode())
        return out

    def q18(self, quantity: str, max_rows: int) -> tuple[np.ndarray, np.ndarray, float]:
        """run_q18's result rows in its own order: (orderkeys, sum_qty_raw, ms)."""
        ok = np.zeros(max(max_rows, 1), np.int32)
        sq = np.zeros(max(max_rows, 1), np.int64)
        ms = C.c_double()
        n = self.lib.ref_q18(self.handle, quantity.encode(), ok.ctypes.data, sq.ctypes.data, max_rows, C.byref(ms))
        if n > max_rows:
            raise RuntimeError(f"run_q18 returned {n} rows, more than the {max_rows} asked for")
        return ok[:n], sq[:n], ms.value

    def q6(self, date: str, discount: str, quantity: str) -> tuple[int, float]:
        r = C.c_int64()
        ms = C.c_double()
        self.lib.ref_q6(self.handle, date.encode(), discount.encode(), quantity.encode(), C.byref(r), C.byref(ms))
        return r.value, ms.value


def parse_trace(text: str) -> dict:
    out = {}
    for line in text.splitlines():
        parts = line.split()
        if len(parts) == 3 and parts[0] in ("COUNT", "PROFILE"):
            out[parts[1]] = int(parts[2])
    return out


def ref_parallel(dbs: list, which: int, delta_days: int = 90, segment: int = 0, date: str = "1993-01-01"):
    """Runs run_q1 (which=1) or run_q3 (which=3) on each database in its own
    thread; returns (wall ms of the slowest, checksum)."""
    lib = dbs[0].lib
    arr = (_P * len(dbs))(*[d.handle for d in dbs])
    cs = C.c_int64()
    ms = lib.ref_parallel(arr, len(dbs), which, delta_days, segment, date.encode(), C.byref(cs))
    return ms, cs.value
