"""Host-side mirror of the reference's per-query API over the GPU engine.

The reference exposes ``run_qN(const Database&, const QNArgs&) -> vector<QNResultRow>``
(bespoke_tpch/query_q1.hpp:22, query_q3.hpp:17, query_q6.hpp:15).  This module
keeps those names, argument meanings and result fields; the work runs in
``libbespoke_gpu.so`` through its C ABI (see ``native.py``).  Errors surface as
:class:`native.BoError` with the engine's status code, the counterpart of the
reference's ``std::runtime_error``.

Inputs are device tensors (torch) or host numpy arrays; the ``*_host`` paths
copy host buffers in and results out inside the call.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import native as N
from .datagen import FLAG_A_LETTERS, FLAG_B_LETTERS, days_from_civil

PRICE_SCALE = 100
DISCOUNT_SCALE = 100


@dataclass
class Q1ResultRow:
    """Fields of the reference's Q1ResultRow (bespoke_tpch/query_q1.hpp:9-20)."""
    returnflag: str
    linestatus: str
    sum_qty: float
    sum_base_price: float
    sum_disc_price: float
    sum_charge: float
    avg_qty: float
    avg_price: float
    avg_disc: float
    count_order: int


def q1_rows_from_aggs(aggs: list[dict], returnflag_dict: list[str], linestatus_dict: list[str]) -> list[Q1ResultRow]:
    """run_q1's finalisation (bespoke_tpch/query_q1.cpp:233-274): groups with a
    non-zero count become rows, integer totals turn into doubles with the same
    expressions (Python floats are IEEE doubles, int->float rounds to nearest as
    the C++ conversion does), then rows are ordered by (returnflag, linestatus)."""
    rows = []
    ls_count = len(linestatus_dict)
    for idx, a in enumerate(aggs):
        if a["count"] == 0:
            continue
        count = float(a["count"])
        sum_qty = float(a["sum_qty"]) / PRICE_SCALE
        sum_base = float(a["sum_base_price"]) / PRICE_SCALE
        rows.append(Q1ResultRow(
            returnflag=returnflag_dict[idx // ls_count],
            linestatus=linestatus_dict[idx % ls_count],
            sum_qty=sum_qty,
            sum_base_price=sum_base,
            sum_disc_price=float(a["sum_disc_price"]) / PRICE_SCALE,
            sum_charge=float(a["sum_charge"]) / (float(PRICE_SCALE) * DISCOUNT_SCALE),
            avg_qty=sum_qty / count,
            avg_price=sum_base / count,
            avg_disc=float(a["sum_disc"]) / DISCOUNT_SCALE / count,
            count_order=a["count"],
        ))
    rows.sort(key=lambda r: (r.returnflag, r.linestatus))
    return rows


def q1_cutoff(delta_days: int) -> int:
    """Absolute-day cutoff of Q1: 1998-12-01 minus DELTA (query_q1.cpp:111-113)."""
    return days_from_civil(1998, 12, 1) - int(delta_days)


def _rows(dev: dict, name: str) -> int:
    """Row count of a device column (torch tensor) of a group-by table set."""
    return int(dev[name].numel())


def _a_id_max(dev: dict, g) -> int:
    """Largest A id: from the device table set when it records it, else from
    the host arrays of ``g``."""
    if "a_id_max" in dev:
        return int(dev["a_id_max"])
    return int(g.a_ids.max()) if len(g.a_ids) else 0


class Engine:
    """One engine context (device, stream, scratch) with the pipeline entry points."""

    def __init__(self, device: int = 0):
        self.ctx = N.Context(device)

    def close(self):
        self.ctx.close()

    @property
    def launches(self) -> int:
        return self.ctx.launches

    def set_stream(self, stream_handle):
        self.ctx.set_stream(stream_handle)

    def synchronize(self):
        self.ctx.synchronize()

    @property
    def host_threads(self) -> int:
        """Host threads of the streamed join's payload gather (0: read in place)."""
        return int(N.lib().bo_host_threads(self.ctx.handle))

    @host_threads.setter
    def host_threads(self, threads: int) -> None:
        self.ctx.call("bo_set_host_threads", int(threads))

    # ------------------------------------------------------------ Q1 -------
    @staticmethod
    def fact_cols(cols, n_rows: int) -> N.FactCols:
        """cols: (ship_date, quantity, ext_price, discount, tax, flag_a, flag_b)."""
        return N.FactCols(*[N.ptr(c) for c in cols], n_rows)

    def q1_fact_device(self, cols, n_rows: int, cutoff: int, n_flag_a: int, n_flag_b: int, out_dev) -> None:
        """Launches the fused scan/filter/group-aggregate on device columns;
        out_dev is a device buffer of >= n_flag_a*n_flag_b bo_q1_agg records."""
        fc = self.fact_cols(cols, n_rows)
        self.ctx.call("bo_q1_fact_device", C.byref(fc), cutoff, n_flag_a, n_flag_b, C.c_void_p(N.ptr(out_dev)))

    def q1_fact_host(self, table, cutoff: int) -> list[dict]:
        """Host arrays in, exact per-group totals out (copies inside the call)."""
        cols = [np.ascontiguousarray(c) for c in table.columns()]
        fc = self.fact_cols(cols, table.n_rows)
        ng = table.n_flag_a * table.n_flag_b
        out = (N.Q1Agg * ng)()
        self.ctx.call("bo_q1_fact_host", C.byref(fc), cutoff, table.n_flag_a, table.n_flag_b, out)
        return [out[g].as_dict() for g in range(ng)]

    def run_q1_fact(self, table, delta_days: int = 90) -> list[Q1ResultRow]:
        """run_q1 over the wide fact layout, flags mapped to order-preserving
        returnflag / linestatus letters."""
        aggs = self.q1_fact_host(table, q1_cutoff(delta_days))
        return q1_rows_from_aggs(aggs, list(FLAG_A_LETTERS[:table.n_flag_a]), list(FLAG_B_LETTERS[:table.n_flag_b]))

    @staticmethod
    def lineitem_cols(li: dict) -> N.LineitemCols:
        names = ["shipdate", "returnflag_linestatus", "extendedprice", "discounted_price", "discount", "tax",
                 "quantity"]
        return N.LineitemCols(*[N.ptr(li.get(k)) for k in names], int(li["n_rows"]))

    def q1_lineitem_host(self, li: dict, cutoff_offset: int, n_groups: int) -> list[dict]:
        lc = self.lineitem_cols(li)
        out = (N.Q1Agg * n_groups)()
        self.ctx.call("bo_q1_lineitem_host", C.byref(lc), cutoff_offset, n_groups, out)
        return [out[g].as_dict() for g in range(n_groups)]

    def q1_lineitem_device(self, li: dict, cutoff_offset: int, n_groups: int, out_dev) -> None:
        lc = self.lineitem_cols(li)
        self.ctx.call("bo_q1_lineitem_device", C.byref(lc), cutoff_offset, n_groups, C.c_void_p(N.ptr(out_dev)))

    def run_q1(self, li: dict, delta_days: int = 90) -> list[Q1ResultRow]:
        """run_q1 (bespoke_tpch/query_q1.cpp:104) over storage-plan lineitem
        columns: ``li`` carries the columns, ``base_date_days`` and the
        returnflag / linestatus dictionaries in code order."""
        cutoff = q1_cutoff(delta_days) - int(li["base_date_days"])
        rf = list(li["returnflag_dict"])
        ls = list(li["linestatus_dict"])
        aggs = self.q1_lineitem_host(li, cutoff, len(rf) * len(ls))
        return q1_rows_from_aggs(aggs, rf, ls)

    # ------------------------------------------------------------ Q6 -------
    def q6_lineitem_host(self, li: dict, start: int, end: int, dmin: int, dmax: int, qlimit: int) -> tuple[int, int]:
        lc = self.lineitem_cols(li)
        out = N.Q6Result()
        self.ctx.call("bo_q6_lineitem_host", C.byref(lc), start, end, dmin, dmax, qlimit, C.byref(out))
        return out.revenue_raw, out.count

    # ----------------------------------------------------------- join ------
    @staticmethod
    def join_cols(build, probe, n_build: int, n_probe: int):
        """build: (key, date, segment); probe: (fk, price, discount)."""
        b = N.JoinBuildCols(*[N.ptr(c) for c in build], n_build)
        p = N.JoinProbeCols(*[N.ptr(c) for c in probe], n_probe)
        return b, p

    def join_plain(self, build, probe, n_build: int, n_probe: int, date_lt: int, seg_eq: int) -> dict:
        """Exact-count pre-pass, one host round trip, build, probe."""
        b, p = self.join_cols(build, probe, n_build, n_probe)
        out = N.JoinResult()
        self.ctx.call("bo_join_plain", C.byref(b), C.byref(p), C.byref(N.JoinParams(date_lt, seg_eq)),
                      C.byref(out))
        return out.as_dict()

    def join_presized(self, build, probe, n_build: int, n_probe: int, date_lt: int, seg_eq: int, pred_dev) -> dict:
        """Table sized on the device from a predicted row count (device float);
        exact rerun if it overflowed."""
        b, p = self.join_cols(build, probe, n_build, n_probe)
        out = N.JoinResult()
        self.ctx.call("bo_join_presized", C.byref(b), C.byref(p), C.byref(N.JoinParams(date_lt, seg_eq)),
                      C.c_void_p(N.ptr(pred_dev)), C.byref(out))
        return out.as_dict()

    def join_presized_device(self, build, probe, n_build: int, n_probe: int, date_lt: int, seg_eq: int, pred_dev,
                             out_dev) -> None:
        b, p = self.join_cols(build, probe, n_build, n_probe)
        self.ctx.call("bo_join_presized_device", C.byref(b), C.byref(p), C.byref(N.JoinParams(date_lt, seg_eq)),
                      C.c_void_p(N.ptr(pred_dev)), C.c_void_p(N.ptr(out_dev)))

    def join_probe_device(self, probe, n_probe: int, out_dev) -> None:
        """Probe the table of this context's last join build with another batch."""
        p = N.JoinProbeCols(*[N.ptr(c) for c in probe], n_probe)
        self.ctx.call("bo_join_probe_device", C.byref(p), C.c_void_p(N.ptr(out_dev)))

    def join_count_device(self, build, n_build: int, date_lt: int, seg_eq: int, count_dev) -> None:
        b = N.JoinBuildCols(*[N.ptr(c) for c in build], n_build)
        self.ctx.call("bo_join_count_device", C.byref(b), C.byref(N.JoinParams(date_lt, seg_eq)),
                      C.c_void_p(N.ptr(count_dev)))

    def join_partitioned(self, build, probe, n_build: int, n_probe: int, date_lt: int, seg_eq: int,
                         log2_partitions: int) -> dict:
        """Radix-partitioned filtered join (2^log2_partitions partitions); the
        plain single pass reruns it if a partition's table was too small."""
        b, p = self.join_cols(build, probe, n_build, n_probe)
        out = N.JoinResult()
        self.ctx.call("bo_join_partitioned", C.byref(b), C.byref(p), C.byref(N.JoinParams(date_lt, seg_eq)),
                      int(log2_partitions), C.byref(out))
        return out.as_dict()

    @staticmethod
    def join_params(params) -> "C.Array":
        """[(date_lt, seg_eq), ...] -> bo_join_params[]."""
        arr = (N.JoinParams * len(params))()
        for i, (d, s) in enumerate(params):
            arr[i] = N.JoinParams(int(d), int(s))
        return arr

    def join_multi(self, build, probe, n_build: int, n_probe: int, params) -> list[dict]:
        """Shared joins over device columns: one count / build / probe pass for
        all (date_lt, seg_eq) pairs in `params`; exact solo reruns if the build
        keys repeat.  Synchronises; one result per pair."""
        b, p = self.join_cols(build, probe, n_build, n_probe)
        prm = self.join_params(params)
        out = (N.JoinResult * len(params))()
        self.ctx.call("bo_join_multi_host", C.byref(b), C.byref(p), prm, len(params), out)
        return [out[i].as_dict() for i in range(len(params))]

    def join_multi_device(self, build, probe, n_build: int, n_probe: int, params, out_dev) -> None:
        """Asynchronous shared joins; out_dev receives len(params) bo_join_result records."""
        b, p = self.join_cols(build, probe, n_build, n_probe)
        self.ctx.call("bo_join_multi_device", C.byref(b), C.byref(p), self.join_params(params), len(params),
                      C.c_void_p(N.ptr(out_dev)))

    def join_host(self, j, mode: int = 0, predicted_rows: float = 0.0) -> dict:
        """Host arrays (a datagen.JoinInput) in; copies inside the call."""
        build = [np.ascontiguousarray(x) for x in (j.b_key, j.b_date, j.b_seg)]
        probe = [np.ascontiguousarray(x) for x in (j.p_fk, j.p_price, j.p_disc)]
        b, p = self.join_cols(build, probe, j.n_build, j.n_probe)
        out = N.JoinResult()
        self.ctx.call("bo_join_host", C.byref(b), C.byref(p), C.byref(N.JoinParams(j.date_lt, j.seg_eq)), mode,
                      float(predicted_rows), C.byref(out))
        return out.as_dict()

    # ------------------------------------------------------- group-by ------
    @staticmethod
    def gb_args(a_id, b_a, b_c, c_cat, c_year, n_a, n_b, n_c, cat_set, year_lo, year_hi, k, a_id_max, a_mask=None):
        cats = np.ascontiguousarray(cat_set, dtype=np.uint16)
        a = N.GbACols(N.ptr(a_id), n_a)
        b = N.GbBCols(N.ptr(b_a), N.ptr(b_c), n_b)
        c = N.GbCCols(N.ptr(c_cat), N.ptr(c_year), n_c)
        prm = N.GbParams(cats.ctypes.data, len(cats), year_lo, year_hi, k, a_id_max, N.ptr(a_mask))
        return a, b, c, prm, cats

    def groupby_plain(self, dev: dict, g) -> dict:
        """Exact distinct pre-pass, one host round trip, aggregation, sort, top-k.
        ``dev`` holds device columns a_ids, b_a, b_c, c_cat, c_year."""
        a, b, c, prm, keep = self.gb_args(dev["a_ids"], dev["b_a"], dev["b_c"], dev["c_cat"], dev["c_year"],
                                          _rows(dev, "a_ids"), _rows(dev, "b_a"), _rows(dev, "c_cat"), g.cat_set, g.year_lo, g.year_hi,
                                          g.k, _a_id_max(dev, g),
                                          dev.get("a_mask"))
        out = N.GbResult()
        self.ctx.call("bo_groupby_topk_plain", C.byref(a), C.byref(b), C.byref(c), C.byref(prm), C.byref(out))
        return out.as_dict()

    def groupby_presized(self, dev: dict, g, pred_dev) -> dict:
        a, b, c, prm, keep = self.gb_args(dev["a_ids"], dev["b_a"], dev["b_c"], dev["c_cat"], dev["c_year"],
                                          _rows(dev, "a_ids"), _rows(dev, "b_a"), _rows(dev, "c_cat"), g.cat_set, g.year_lo, g.year_hi,
                                          g.k, _a_id_max(dev, g),
                                          dev.get("a_mask"))
        out = N.GbResult()
        self.ctx.call("bo_groupby_topk_presized", C.byref(a), C.byref(b), C.byref(c), C.byref(prm),
                      C.c_void_p(N.ptr(pred_dev)), C.byref(out))
        return out.as_dict()

    def groupby_presized_device(self, dev: dict, g, pred_dev, out_dev) -> None:
        a, b, c, prm, keep = self.gb_args(dev["a_ids"], dev["b_a"], dev["b_c"], dev["c_cat"], dev["c_year"],
                                          _rows(dev, "a_ids"), _rows(dev, "b_a"), _rows(dev, "c_cat"), g.cat_set, g.year_lo, g.year_hi,
                                          g.k, _a_id_max(dev, g),
                                          dev.get("a_mask"))
        self.ctx.call("bo_groupby_topk_presized_device", C.byref(a), C.byref(b), C.byref(c), C.byref(prm),
                      C.c_void_p(N.ptr(pred_dev)), C.c_void_p(N.ptr(out_dev)))

    def groupby_partitioned(self, dev: dict, g, log2_partitions: int, predicted_joined_rows: float) -> dict:
        """Radix-partitioned form: 2^log2_partitions partitions sized from the
        predicted joined rows; plain rerun if a partition was too small."""
        a, b, c, prm, keep = self.gb_args(dev["a_ids"], dev["b_a"], dev["b_c"], dev["c_cat"], dev["c_year"],
                                          _rows(dev, "a_ids"), _rows(dev, "b_a"), _rows(dev, "c_cat"), g.cat_set, g.year_lo, g.year_hi,
                                          g.k, _a_id_max(dev, g), dev.get("a_mask"))
        out = N.GbResult()
        self.ctx.call("bo_groupby_topk_partitioned", C.byref(a), C.byref(b), C.byref(c), C.byref(prm),
                      int(log2_partitions), float(predicted_joined_rows), C.byref(out))
        return out.as_dict()

    def groupby_partitioned_device(self, dev: dict, g, log2_partitions: int, predicted_joined_rows: float,
                                   out_dev) -> None:
        a, b, c, prm, keep = self.gb_args(dev["a_ids"], dev["b_a"], dev["b_c"], dev["c_cat"], dev["c_year"],
                                          _rows(dev, "a_ids"), _rows(dev, "b_a"), _rows(dev, "c_cat"), g.cat_set, g.year_lo, g.year_hi,
                                          g.k, _a_id_max(dev, g), dev.get("a_mask"))
        self.ctx.call("bo_groupby_topk_partitioned_device", C.byref(a), C.byref(b), C.byref(c), C.byref(prm),
                      int(log2_partitions), float(predicted_joined_rows), C.c_void_p(N.ptr(out_dev)))

    def groupby_distinct_device(self, dev: dict, g, out_dev) -> None:
        a, b, c, prm, keep = self.gb_args(dev["a_ids"], dev["b_a"], dev["b_c"], dev["c_cat"], dev["c_year"],
                                          _rows(dev, "a_ids"), _rows(dev, "b_a"), _rows(dev, "c_cat"), g.cat_set, g.year_lo, g.year_hi,
                                          g.k, _a_id_max(dev, g),
                                          dev.get("a_mask"))
        self.ctx.call("bo_groupby_distinct_device", C.byref(a), C.byref(b), C.byref(c), C.byref(prm),
                      C.c_void_p(N.ptr(out_dev)))

    def groupby_to_device(self, g, prebuild_a_mask: bool = False) -> dict:
        """Uploads the three tables; optionally builds A's id mask once (a
        per-table structure, like the sketches)."""
        import torch

        d = {k: torch.from_numpy(np.ascontiguousarray(getattr(g, k))).cuda()
             for k in ("a_ids", "b_a", "b_c", "c_cat", "c_year")}
        d["a_id_max"] = int(g.a_ids.max()) if len(g.a_ids) else 0
        if prebuild_a_mask:
            m = torch.zeros((d["a_id_max"] + 32) // 32, dtype=torch.int32, device="cuda")
            a = N.GbACols(N.ptr(d["a_ids"]), len(g.a_ids))
            self.ctx.call("bo_groupby_a_mask_device", C.byref(a), d["a_id_max"], C.c_void_p(m.data_ptr()))
            d["a_mask"] = m
        return d

    # ---------------------------------------------------------- sort -------
    def radix_sort_pairs_host(self, keys: np.ndarray, vals: np.ndarray, begin_bit: int = 0, end_bit: int = 64):
        k = np.ascontiguousarray(keys, dtype=np.uint64).copy()
        v = np.ascontiguousarray(vals, dtype=np.uint32).copy()
        self.ctx.call("bo_radix_sort_pairs_host", C.c_void_p(k.ctypes.data), C.c_void_p(v.ctypes.data), len(k),
                      begin_bit, end_bit)
        return k, v


class PinnedColumns:
    """numpy arrays copied into pinned, mapped host buffers (the inputs of the
    streamed entry points); freed with close()."""

    def __init__(self, engine: Engine, arrays: dict):
        self.engine = engine
        self.ptrs = {}
        for name, a in arrays.items():
            a = np.ascontiguousarray(a)
            h = C.c_void_p()
            engine.ctx.call("bo_host_alloc_pinned", C.c_size_t(max(a.nbytes, 64)), C.byref(h))
            if a.nbytes:
                C.memmove(h.value, a.ctypes.data, a.nbytes)
            self.ptrs[name] = h.value

    def close(self):
        for p in self.ptrs.values():
            self.engine.ctx.call("bo_host_free_pinned", C.c_void_p(p))
        self.ptrs.clear()


def join_stream(engine: Engine, pc: PinnedColumns, n_build: int, n_probe: int, date_lt: int, seg_eq: int,
                pred_dev=None) -> dict:
    """bo_join_stream_host over pinned columns named b_key, b_date, b_seg,
    p_fk, p_price, p_disc."""
    p = pc.ptrs
    b = N.JoinBuildCols(p["b_key"], p["b_date"], p["b_seg"], n_build)
    pr = N.JoinProbeCols(p["p_fk"], p["p_price"], p["p_disc"], n_probe)
    out = N.JoinResult()
    engine.ctx.call("bo_join_stream_host", C.byref(b), C.byref(pr), C.byref(N.JoinParams(date_lt, seg_eq)),
                    C.c_void_p(N.ptr(pred_dev)), C.byref(out))
    return out.as_dict()


def join_stream_async(engine: Engine, pc: PinnedColumns, n_build: int, n_probe: int, date_lt: int, seg_eq: int,
                      pred_dev, out_pinned_addr: int) -> None:
    """bo_join_stream_host_async: enqueue one presized streamed join whose
    result lands at out_pinned_addr (pinned host memory) after a synchronize."""
    p = pc.ptrs
    b = N.JoinBuildCols(p["b_key"], p["b_date"], p["b_seg"], n_build)
    pr = N.JoinProbeCols(p["p_fk"], p["p_price"], p["p_disc"], n_probe)
    engine.ctx.call("bo_join_stream_host_async", C.byref(b), C.byref(pr), C.byref(N.JoinParams(date_lt, seg_eq)),
                    C.c_void_p(N.ptr(pred_dev)), C.c_void_p(out_pinned_addr))
