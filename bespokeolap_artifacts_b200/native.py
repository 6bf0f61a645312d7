"""ctypes binding of ``libbespoke_gpu.so`` (the C ABI in ``include/bespoke_gpu.h``).

The library is the only compute path: if it is missing or was not built, every
entry point raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libbespoke_gpu.so"

BO_OK = 0
BO_ERR_OVERFLOW = -3
BO_ERR_DATA = -6
STATUS_NAMES = {
    0: "BO_OK",
    -1: "BO_ERR_INVALID",
    -2: "BO_ERR_OOM",
    -3: "BO_ERR_OVERFLOW",
    -4: "BO_ERR_TIMEOUT",
    -5: "BO_ERR_CUDA",
    -6: "BO_ERR_DATA",
    -7: "BO_ERR_UNSUPPORTED",
}

Q1_MAX_GROUPS = 8


class BoError(RuntimeError):
    """A failed call into the engine; ``status`` is the BO_ERR_* code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


# ----------------------------------------------------------------- structs --
class I128(C.Structure):
    _fields_ = [("lo", C.c_uint64), ("hi", C.c_int64)]

    def value(self) -> int:
        return (self.hi << 64) | self.lo


class Q1Agg(C.Structure):
    _fields_ = [
        ("count", C.c_int64),
        ("sum_qty", C.c_int64),
        ("sum_base_price", C.c_int64),
        ("sum_disc", C.c_int64),
        ("sum_disc_price", C.c_int64),
        ("sum_disc_price_exact", C.c_int64),
        ("sum_charge", I128),
        ("sum_charge_exact", I128),
    ]

    def as_dict(self) -> dict:
        return {
            "count": self.count,
            "sum_qty": self.sum_qty,
            "sum_base_price": self.sum_base_price,
            "sum_disc": self.sum_disc,
            "sum_disc_price": self.sum_disc_price,
            "sum_disc_price_exact": self.sum_disc_price_exact,
            "sum_charge": self.sum_charge.value(),
            "sum_charge_exact": self.sum_charge_exact.value(),
        }


class FactCols(C.Structure):
    _fields_ = [
        ("ship_date", C.c_void_p),
        ("quantity", C.c_void_p),
        ("ext_price", C.c_void_p),
        ("discount", C.c_void_p),
        ("tax", C.c_void_p),
        ("flag_a", C.c_void_p),
        ("flag_b", C.c_void_p),
        ("n_rows", C.c_int64),
    ]


class LineitemCols(C.Structure):
    _fields_ = [
        ("shipdate", C.c_void_p),
        ("returnflag_linestatus", C.c_void_p),
        ("extendedprice", C.c_void_p),
        ("discounted_price", C.c_void_p),
        ("discount", C.c_void_p),
        ("tax", C.c_void_p),
        ("quantity", C.c_void_p),
        ("n_rows", C.c_int64),
    ]


class Q6Result(C.Structure):
    _fields_ = [("revenue_raw", C.c_int64), ("count", C.c_int64)]


class JoinBuildCols(C.Structure):
    _fields_ = [("key", C.c_void_p), ("date", C.c_void_p), ("segment", C.c_void_p), ("n_rows", C.c_int64)]


class JoinProbeCols(C.Structure):
    _fields_ = [("fk", C.c_void_p), ("price", C.c_void_p), ("discount", C.c_void_p), ("n_rows", C.c_int64)]


class JoinParams(C.Structure):
    _fields_ = [("date_lt", C.c_int32), ("segment_eq", C.c_int32)]


JOIN_MULTI_MAX = 32
GB_MAX_LOG2_PARTITIONS = 14
JOIN_MAX_LOG2_PARTITIONS = 14


class JoinResult(C.Structure):
    _fields_ = [
        ("build_rows", C.c_int64), ("distinct_keys", C.c_int64), ("match_count", C.c_int64),
        ("sum_exact", I128), ("sum_trunc", I128), ("capacity_log2", C.c_int32), ("overflowed", C.c_int32),
        ("reruns", C.c_int32), ("mode", C.c_int32),
    ]

    def as_dict(self) -> dict:
        return dict(build_rows=self.build_rows, distinct_keys=self.distinct_keys, match_count=self.match_count,
                    sum_exact=self.sum_exact.value(), sum_trunc=self.sum_trunc.value(),
                    capacity_log2=self.capacity_log2, overflowed=self.overflowed, reruns=self.reruns,
                    mode=self.mode)


GB_MAX_K = 64


class GbACols(C.Structure):
    _fields_ = [("id", C.c_void_p), ("n_rows", C.c_int64)]


class GbBCols(C.Structure):
    _fields_ = [("a_id", C.c_void_p), ("c_id", C.c_void_p), ("n_rows", C.c_int64)]


class GbCCols(C.Structure):
    _fields_ = [("category", C.c_void_p), ("year", C.c_void_p), ("n_rows", C.c_int64)]


class GbParams(C.Structure):
    _fields_ = [("categories", C.c_void_p), ("n_categories", C.c_int32), ("year_lo", C.c_int32),
                ("year_hi", C.c_int32), ("k", C.c_int32), ("a_id_max", C.c_int32), ("a_mask", C.c_void_p)]


class GbRow(C.Structure):
    _fields_ = [("a_id", C.c_int32), ("min_year", C.c_int32), ("count", C.c_int64)]


class GbResult(C.Structure):
    _fields_ = [("n_groups", C.c_int64), ("joined_rows", C.c_int64), ("c_qualifying", C.c_int64),
                ("exact_distinct", C.c_int64), ("capacity_log2", C.c_int32), ("overflowed", C.c_int32),
                ("reruns", C.c_int32), ("mode", C.c_int32), ("n_rows_out", C.c_int32), ("pad", C.c_int32),
                ("rows", GbRow * GB_MAX_K)]

    def as_dict(self) -> dict:
        n = self.n_rows_out
        return dict(n_groups=self.n_groups, joined_rows=self.joined_rows, c_qualifying=self.c_qualifying,
                    exact_distinct=self.exact_distinct, capacity_log2=self.capacity_log2,
                    overflowed=self.overflowed, reruns=self.reruns, mode=self.mode,
                    keys=[self.rows[i].a_id for i in range(n)], counts=[self.rows[i].count for i in range(n)],
                    min_years=[self.rows[i].min_year for i in range(n)])


class TpchQ3Tables(C.Structure):
    """``bo_tpch_q3_tables``: storage-plan columns of customer, orders, lineitem."""
    _fields_ = [("c_custkey", C.c_void_p), ("c_mktsegment", C.c_void_p), ("n_customer", C.c_int64),
                ("custkey_bound", C.c_int32), ("pad0", C.c_int32), ("o_orderkey", C.c_void_p),
                ("o_custkey", C.c_void_p), ("o_orderdate", C.c_void_p), ("o_shippriority", C.c_void_p),
                ("n_orders", C.c_int64), ("orderkey_to_row", C.c_void_p), ("n_orderkey_map", C.c_int64),
                ("l_orderkey", C.c_void_p), ("l_shipdate", C.c_void_p), ("l_discounted_price", C.c_void_p),
                ("n_lineitem", C.c_int64)]


class TpchQ3Row(C.Structure):
    _fields_ = [("revenue_raw", C.c_int64), ("orderkey", C.c_int32), ("shippriority", C.c_int32),
                ("orderdate_offset", C.c_int16), ("pad0", C.c_int16), ("pad1", C.c_int32)]


class TpchQ10Tables(C.Structure):
    """``bo_tpch_q10_tables``: orders with lineitem ranges, lineitem, customer map and nations."""
    _fields_ = [("o_orderkey", C.c_void_p), ("o_custkey", C.c_void_p), ("o_orderdate", C.c_void_p),
                ("o_li_begin", C.c_void_p), ("o_li_end", C.c_void_p), ("n_orders", C.c_int64),
                ("l_orderkey", C.c_void_p), ("l_returnflag_linestatus", C.c_void_p),
                ("l_discounted_price", C.c_void_p), ("n_lineitem", C.c_int64),
                ("lineitem_orderkey_sorted", C.c_int32), ("nation_bound", C.c_int32),
                ("custkey_to_row", C.c_void_p), ("n_custkey_map", C.c_int64), ("c_nationkey", C.c_void_p),
                ("n_customer", C.c_int64), ("c_name_offsets", C.c_void_p), ("c_address_offsets", C.c_void_p),
                ("c_phone_offsets", C.c_void_p), ("c_comment_offsets", C.c_void_p), ("c_acctbal", C.c_void_p)]


class TpchQ10Row(C.Structure):
    _fields_ = [("revenue_raw", C.c_int64), ("custkey", C.c_int32), ("cust_row", C.c_int32),
                ("nationkey", C.c_int32), ("acctbal_raw", C.c_int32),
                ("name_begin", C.c_uint32), ("name_len", C.c_uint32), ("address_begin", C.c_uint32),
                ("address_len", C.c_uint32), ("phone_begin", C.c_uint32), ("phone_len", C.c_uint32),
                ("comment_begin", C.c_uint32), ("comment_len", C.c_uint32)]


class TpchQ18Tables(C.Structure):
    """``bo_tpch_q18_tables``: orders, lineitem quantities, customer map, key-layout flags."""
    _fields_ = [("o_orderkey", C.c_void_p), ("o_custkey", C.c_void_p), ("o_orderdate", C.c_void_p),
                ("o_totalprice", C.c_void_p), ("n_orders", C.c_int64), ("l_orderkey", C.c_void_p),
                ("l_quantity", C.c_void_p), ("n_lineitem", C.c_int64), ("custkey_to_row", C.c_void_p),
                ("n_custkey_map", C.c_int64), ("n_customer", C.c_int64), ("orderkey_bound", C.c_int64),
                ("dense_orderkeys", C.c_int32), ("dense_custkeys", C.c_int32)]


class TpchQ18Row(C.Structure):
    _fields_ = [("sum_qty_raw", C.c_int64), ("custkey", C.c_int32), ("cust_row", C.c_int32),
                ("orderkey", C.c_int32), ("totalprice_raw", C.c_int32), ("orderdate_offset", C.c_int16),
                ("pad0", C.c_int16), ("pad1", C.c_int32)]


class TpchQ4Tables(C.Structure):
    """``bo_tpch_q4_tables``: date-sorted orders (keys, dates, priorities, lineitem ranges), lineitem keys and
    packed commit / receipt dates."""
    _fields_ = [("o_orderkey", C.c_void_p), ("o_orderdate", C.c_void_p), ("o_orderpriority", C.c_void_p),
                ("o_li_begin", C.c_void_p), ("o_li_end", C.c_void_p), ("n_orders", C.c_int64),
                ("l_orderkey", C.c_void_p), ("l_commit_receipt", C.c_void_p), ("n_lineitem", C.c_int64),
                ("lineitem_orderkey_sorted", C.c_int32), ("n_priorities", C.c_int32)]


class TpchQ5Tables(C.Structure):
    """``bo_tpch_q5_tables``: date-sorted orders (keys, dates, customer nations, lineitem ranges), lineitem keys,
    supplier nations and discounted prices."""
    _fields_ = [("o_orderkey", C.c_void_p), ("o_orderdate", C.c_void_p), ("o_cust_nation", C.c_void_p),
                ("o_li_begin", C.c_void_p), ("o_li_end", C.c_void_p), ("n_orders", C.c_int64),
                ("l_orderkey", C.c_void_p), ("l_supp_nation", C.c_void_p), ("l_discounted_price", C.c_void_p),
                ("n_lineitem", C.c_int64), ("lineitem_orderkey_sorted", C.c_int32), ("n_nations", C.c_int32)]


class TpchQ7Tables(C.Structure):
    """``bo_tpch_q7_tables``: lineitem shipdates, suppkeys, orderkeys, discounted prices; the orderkey map and
    orders' customer nations."""
    _fields_ = [("l_shipdate", C.c_void_p), ("l_suppkey", C.c_void_p), ("l_orderkey", C.c_void_p),
                ("l_discounted_price", C.c_void_p), ("n_lineitem", C.c_int64), ("orderkey_to_row", C.c_void_p),
                ("n_orderkey_map", C.c_int64), ("o_cust_nation", C.c_void_p), ("n_orders", C.c_int64)]


class TpchQ8Tables(C.Structure):
    """``bo_tpch_q8_tables``: lineitem part/supp/order keys, prices, discounts; the orderkey map, orders'
    custkeys and dates; customer keys and nations; part keys and type codes."""
    _fields_ = [("l_partkey", C.c_void_p), ("l_suppkey", C.c_void_p), ("l_orderkey", C.c_void_p),
                ("l_extendedprice", C.c_void_p), ("l_discount", C.c_void_p), ("n_lineitem", C.c_int64),
                ("orderkey_to_row", C.c_void_p), ("n_orderkey_map", C.c_int64), ("o_custkey", C.c_void_p),
                ("o_orderdate", C.c_void_p), ("n_orders", C.c_int64), ("c_custkey", C.c_void_p),
                ("c_nationkey", C.c_void_p), ("n_customer", C.c_int64), ("max_custkey", C.c_int32),
                ("max_partkey", C.c_int32), ("p_partkey", C.c_void_p), ("p_type", C.c_void_p), ("n_part", C.c_int64)]


class TpchQ22Tables(C.Structure):
    """``bo_tpch_q22_tables``: customer keys, balances, phone classes; the per-custkey order bits."""
    _fields_ = [("c_custkey", C.c_void_p), ("c_acctbal", C.c_void_p), ("c_phone_prefix", C.c_void_p),
                ("c_phone_pair", C.c_void_p), ("n_customer", C.c_int64), ("o_has_order", C.c_void_p),
                ("n_order_custkeys", C.c_int64)]


class TpchQ11Tables(C.Structure):
    """``bo_tpch_q11_tables``: partsupp rows by partkey (partkeys, suppkeys, values) and the partkey range."""
    _fields_ = [("ps_partkey", C.c_void_p), ("ps_suppkey", C.c_void_p), ("ps_value", C.c_void_p),
                ("n_partsupp", C.c_int64), ("min_partkey", C.c_int32), ("max_partkey", C.c_int32)]


class TpchQ15Tables(C.Structure):
    """``bo_tpch_q15_tables``: lineitem shipdates, suppkeys, discounted prices."""
    _fields_ = [("l_shipdate", C.c_void_p), ("l_suppkey", C.c_void_p), ("l_discounted_price", C.c_void_p),
                ("n_lineitem", C.c_int64)]


class TpchQ17Tables(C.Structure):
    """``bo_tpch_q17_tables``: lineitem partkeys, quantities, extended prices; part keys, brand and container
    codes; the largest part key."""
    _fields_ = [("l_partkey", C.c_void_p), ("l_quantity", C.c_void_p), ("l_extendedprice", C.c_void_p),
                ("n_lineitem", C.c_int64), ("p_partkey", C.c_void_p), ("p_brand", C.c_void_p),
                ("p_container", C.c_void_p), ("n_part", C.c_int64), ("max_partkey", C.c_int32), ("pad", C.c_int32)]


class TpchQ9Tables(C.Structure):
    """``bo_tpch_q9_tables``: lineitem partkeys, suppkeys, orderkeys, quantities, discounted prices and
    supplier nations; part names (bytes + offsets) and keys; partsupp suppkeys and supply costs sorted by
    partkey with per-key row offsets; the per-orderkey year table."""
    _fields_ = [("l_partkey", C.c_void_p), ("l_suppkey", C.c_void_p), ("l_orderkey", C.c_void_p),
                ("l_quantity", C.c_void_p), ("l_discounted_price", C.c_void_p), ("l_supp_nation", C.c_void_p),
                ("n_lineitem", C.c_int64), ("p_name", C.c_void_p), ("p_name_offsets", C.c_void_p),
                ("p_partkey", C.c_void_p), ("n_part", C.c_int64), ("ps_suppkey", C.c_void_p),
                ("ps_supplycost", C.c_void_p), ("ps_part_begin", C.c_void_p), ("n_part_keys", C.c_int64),
                ("slots_per_part", C.c_int32), ("pad", C.c_int32), ("o_year_by_key", C.c_void_p),
                ("n_orderkeys", C.c_int64)]


class TpchQ19Tables(C.Structure):
    """``bo_tpch_q19_tables``: lineitem ship-mode and ship-instruct codes, partkeys, quantities, prices and
    discounts; the last part row per key, part brand / container codes and sizes; the mask's key count."""
    _fields_ = [("l_shipmode", C.c_void_p), ("l_shipinstruct", C.c_void_p), ("l_partkey", C.c_void_p),
                ("l_quantity", C.c_void_p), ("l_extendedprice", C.c_void_p), ("l_discount", C.c_void_p),
                ("n_lineitem", C.c_int64), ("p_row_by_key", C.c_void_p), ("n_part_keys", C.c_int64),
                ("p_brand", C.c_void_p), ("p_container", C.c_void_p), ("p_size", C.c_void_p), ("n_part", C.c_int64),
                ("n_mask", C.c_int64)]


class TpchQ21Tables(C.Structure):
    """``bo_tpch_q21_tables``: lineitem orderkeys, suppkeys, packed commit / receipt dates; date-sorted orders'
    keys, status codes and lineitem ranges; whether lineitems are sorted by orderkey."""
    _fields_ = [("l_orderkey", C.c_void_p), ("l_suppkey", C.c_void_p), ("l_commit_receipt", C.c_void_p),
                ("n_lineitem", C.c_int64), ("o_orderkey", C.c_void_p), ("o_orderstatus", C.c_void_p),
                ("o_li_begin", C.c_void_p), ("o_li_end", C.c_void_p), ("n_orders", C.c_int64),
                ("lineitem_orderkey_sorted", C.c_int32), ("pad", C.c_int32)]


class CebCol(C.Structure):
    """``bo_ceb_col``: int32 values (string columns: dictionary codes) and an optional null byte per row."""
    _fields_ = [("values", C.c_void_p), ("is_null", C.c_void_p)]


class CebQ1aTables(C.Structure):
    """``bo_ceb_q1a_tables``: the columns CEB query 1a reads, in the reference's column layout."""
    _fields_ = [("t_id", CebCol), ("t_kind_id", CebCol), ("t_year", CebCol), ("n_title", C.c_int64),
                ("max_title_id", C.c_int32), ("pad0", C.c_int32),
                ("mi_movie_id", CebCol), ("mi_info_type_id", CebCol), ("mi_info", CebCol), ("n_movie_info", C.c_int64),
                ("ci_movie_id", CebCol), ("ci_person_id", CebCol), ("ci_role_id", CebCol), ("n_cast_info", C.c_int64),
                ("kt_id", CebCol), ("kt_kind", CebCol), ("n_kind_type", C.c_int64),
                ("rt_id", CebCol), ("rt_role", CebCol), ("n_role_type", C.c_int64),
                ("nm_id", CebCol), ("nm_gender", CebCol), ("n_name", C.c_int64)]


class CebQ1aParams(C.Structure):
    """``bo_ceb_q1a_params``: years, the info-type filter and the per-code byte arrays (host memory)."""
    _fields_ = [("year1", C.c_int32), ("year2", C.c_int32), ("info_type_filter", C.c_void_p),
                ("info_type_size", C.c_int32), ("n_info_codes", C.c_int32), ("info_match", C.c_void_p),
                ("kind_allowed", C.c_void_p), ("role_allowed", C.c_void_p), ("gender_allowed", C.c_void_p),
                ("n_kind_codes", C.c_int32), ("n_role_codes", C.c_int32), ("n_gender_codes", C.c_int32),
                ("kind_mask_size", C.c_int32), ("role_mask_size", C.c_int32), ("person_mask_size", C.c_int32),
                ("pad", C.c_int32)]


class CebDict(C.Structure):
    """``bo_ceb_dict``: a string dictionary on the device (bytes, n + 1 offsets, each code's string rank)."""
    _fields_ = [("bytes", C.c_void_p), ("offsets", C.c_void_p), ("rank", C.c_void_p), ("n", C.c_int64)]


class CebQ3bTables(C.Structure):
    """``bo_ceb_q3b_tables``: the columns CEB query 3b reads, its string dictionaries and id bounds."""
    _fields_ = [("kt_id", CebCol), ("kt_kind", CebCol), ("n_kind_type", C.c_int64),
                ("rt_id", CebCol), ("rt_role", CebCol), ("n_role_type", C.c_int64),
                ("cn_id", CebCol), ("cn_name", CebCol), ("n_company_name", C.c_int64),
                ("mc_movie_id", CebCol), ("mc_company_id", CebCol), ("mc_company_type_id", CebCol),
                ("n_movie_companies", C.c_int64),
                ("mk_movie_id", CebCol), ("mk_keyword_id", CebCol), ("n_movie_keyword", C.c_int64),
                ("t_id", CebCol), ("t_title", CebCol), ("t_kind_id", CebCol), ("n_title", C.c_int64),
                ("ci_movie_id", CebCol), ("ci_person_id", CebCol), ("ci_role_id", CebCol), ("n_cast_info", C.c_int64),
                ("nm_id", CebCol), ("nm_name", CebCol), ("nm_pcode", CebCol), ("n_name", C.c_int64),
                ("title_dict", CebDict), ("name_dict", CebDict), ("company_dict", CebDict), ("pcode_dict", CebDict),
                ("movie_bound", C.c_int32), ("person_bound", C.c_int32)]


class CebQ3bParams(C.Structure):
    """``bo_ceb_q3b_params``: kind / role codes, id mask sizes and the three ILIKE patterns (host memory)."""
    _fields_ = [("kind_allowed", C.c_void_p), ("role_allowed", C.c_void_p), ("n_kind_codes", C.c_int32),
                ("n_role_codes", C.c_int32), ("kind_mask_size", C.c_int32), ("role_mask_size", C.c_int32),
                ("company_map_size", C.c_int32), ("title_type", C.c_int32), ("pcode_type", C.c_int32),
                ("company_type", C.c_int32), ("title_pat", C.c_void_p), ("pcode_pat", C.c_void_p),
                ("company_pat", C.c_void_p), ("title_len", C.c_int32), ("pcode_len", C.c_int32),
                ("company_len", C.c_int32), ("pad", C.c_int32)]


class CebQ3bRow(C.Structure):
    _fields_ = [("title_code", C.c_int32), ("name_code", C.c_int32), ("company_code", C.c_int32),
                ("pad", C.c_int32), ("count", C.c_int64)]


class CebQ10aTables(C.Structure):
    """``bo_ceb_q10a_tables``: the columns CEB query 10a reads and the name dictionary on the device."""
    _fields_ = [("t_id", CebCol), ("t_kind_id", CebCol), ("t_year", CebCol), ("n_title", C.c_int64),
                ("mi_movie_id", CebCol), ("mi_info_type_id", CebCol), ("mi_info", CebCol), ("n_movie_info", C.c_int64),
                ("ci_movie_id", CebCol), ("ci_person_id", CebCol), ("ci_role_id", CebCol), ("n_cast_info", C.c_int64),
                ("kt_id", CebCol), ("kt_kind", CebCol), ("n_kind_type", C.c_int64),
                ("rt_id", CebCol), ("rt_role", CebCol), ("n_role_type", C.c_int64),
                ("nm_id", CebCol), ("nm_name", CebCol), ("n_name", C.c_int64),
                ("name_dict", C.c_void_p), ("name_dict_offsets", C.c_void_p), ("n_name_codes", C.c_int64)]


class CebQ10aParams(C.Structure):
    """``bo_ceb_q10a_params``: the info-type mask, dense info indices per code, kind / role codes and the
    ILIKE pattern (host memory)."""
    _fields_ = [("info_type_mask", C.c_void_p), ("info_type_size", C.c_int32), ("n_info_codes", C.c_int32),
                ("info_dense", C.c_void_p), ("n_info_dense", C.c_int32), ("n_kind_codes", C.c_int32),
                ("kind_allowed", C.c_void_p), ("role_allowed", C.c_void_p), ("n_role_codes", C.c_int32),
                ("pattern_type", C.c_int32), ("pattern", C.c_void_p), ("pattern_len", C.c_int32), ("pad", C.c_int32)]


class CebQ10aRow(C.Structure):
    _fields_ = [("name_code", C.c_int32), ("info_dense", C.c_int32), ("has_year", C.c_int32),
                ("min_year", C.c_int32), ("max_year", C.c_int32)]


class TpchQ14Tables(C.Structure):
    """``bo_tpch_q14_tables``: lineitem shipdates, partkeys, discounted prices; the part promo flag per key."""
    _fields_ = [("l_shipdate", C.c_void_p), ("l_partkey", C.c_void_p), ("l_discounted_price", C.c_void_p),
                ("n_lineitem", C.c_int64), ("p_promo_by_key", C.c_void_p), ("n_promo_map", C.c_int64)]


class TpchQ12Tables(C.Structure):
    """``bo_tpch_q12_tables``: lineitem ship modes, packed commit / receipt dates, shipdates, orderkeys,
    optional shard maxima; orders map and priorities."""
    _fields_ = [("l_shipmode", C.c_void_p), ("l_commit_receipt", C.c_void_p), ("l_shipdate", C.c_void_p),
                ("l_orderkey", C.c_void_p), ("l_shard_max_shipdate", C.c_void_p), ("n_lineitem", C.c_int64),
                ("orderkey_to_row", C.c_void_p), ("n_orderkey_map", C.c_int64), ("o_orderpriority", C.c_void_p),
                ("n_orders", C.c_int64)]


class TpchQ16Tables(C.Structure):
    """``bo_tpch_q16_tables``: part keys, brand / type codes, sizes; partsupp (by partkey); supplier flags."""
    _fields_ = [("p_partkey", C.c_void_p), ("p_brand", C.c_void_p), ("p_type", C.c_void_p), ("p_size", C.c_void_p),
                ("n_part", C.c_int64), ("ps_partkey", C.c_void_p), ("ps_suppkey", C.c_void_p),
                ("n_partsupp", C.c_int64), ("s_banned", C.c_void_p), ("n_banned", C.c_int64)]


class TpchQ16Params(C.Structure):
    """``bo_tpch_q16_params``: size mask, banned brand, rows per part, dictionary ranks (host arrays)."""
    _fields_ = [("size_mask", C.c_uint64), ("banned_brand", C.c_int32), ("rows_per_part", C.c_int32),
                ("n_brand", C.c_int32), ("n_type", C.c_int32), ("brand_rank", C.c_void_p),
                ("type_rank", C.c_void_p), ("type_banned", C.c_void_p)]


class TpchQ16Row(C.Structure):
    _fields_ = [("brand_code", C.c_int32), ("type_code", C.c_int32), ("size", C.c_int32), ("pad", C.c_int32),
                ("supplier_cnt", C.c_int64)]


class TpchQ20Tables(C.Structure):
    """``bo_tpch_q20_tables``: part keys and names; lineitem ship dates, keys, supplier nations, quantities;
    partsupp (by partkey) with availqty and per-partkey offsets; supplier nations by key, rows in name order."""
    _fields_ = [("p_partkey", C.c_void_p), ("p_name", C.c_void_p), ("p_name_offsets", C.c_void_p),
                ("n_part", C.c_int64), ("max_partkey", C.c_int32), ("max_suppkey", C.c_int32),
                ("l_shipdate", C.c_void_p), ("l_partkey", C.c_void_p), ("l_suppkey", C.c_void_p),
                ("l_supp_nation", C.c_void_p), ("l_quantity", C.c_void_p), ("n_lineitem", C.c_int64),
                ("ps_partkey", C.c_void_p), ("ps_suppkey", C.c_void_p), ("ps_availqty", C.c_void_p),
                ("n_partsupp", C.c_int64), ("ps_part_begin", C.c_void_p), ("n_ps_part_keys", C.c_int64),
                ("s_nation_by_key", C.c_void_p), ("s_suppkey", C.c_void_p), ("s_nationkey", C.c_void_p),
                ("s_row_by_name", C.c_void_p), ("n_supplier", C.c_int64)]


class TpchQ2Tables(C.Structure):
    """``bo_tpch_q2_tables``: part sizes, type and manufacturer codes; partsupp suppkeys and costs with
    per-partkey offsets; supplier nation indexes and order ranks."""
    _fields_ = [("p_size", C.c_void_p), ("p_type", C.c_void_p), ("p_mfgr", C.c_void_p), ("n_part", C.c_int64),
                ("ps_suppkey", C.c_void_p), ("ps_supplycost", C.c_void_p), ("n_partsupp", C.c_int64),
                ("ps_part_begin", C.c_void_p), ("n_ps_part_keys", C.c_int64), ("s_nation_idx", C.c_void_p),
                ("s_rank", C.c_void_p), ("n_supplier", C.c_int64)]


class TpchQ2Row(C.Structure):
    _fields_ = [("partkey", C.c_int32), ("supplier_row", C.c_int32), ("mfgr_code", C.c_int32), ("pad", C.c_int32)]


class TpchQ11Row(C.Structure):
    _fields_ = [("ps_partkey", C.c_int32), ("pad", C.c_int32), ("value_raw", C.c_int64)]


class HostStr(C.Structure):
    _fields_ = [("ptr", C.c_void_p), ("len", C.c_uint64)]


class TpchQ10HostStrings(C.Structure):
    """``bo_tpch_q10_host_strings``: host bytes of the customer name / address / phone / comment columns and the
    nation names by key."""
    _fields_ = [("name_data", C.c_void_p), ("address_data", C.c_void_p), ("phone_data", C.c_void_p),
                ("comment_data", C.c_void_p), ("nation_names", C.c_void_p), ("n_nation", C.c_int32),
                ("pad", C.c_int32)]


class TpchQ10HostRow(C.Structure):
    _fields_ = [("custkey", C.c_int32), ("acctbal_raw", C.c_int32), ("revenue_raw", C.c_int64),
                ("name", HostStr), ("nation_name", HostStr), ("address", HostStr), ("phone", HostStr),
                ("comment", HostStr)]


class TpchQ13Tables(C.Structure):
    """``bo_tpch_q13_tables``: order comments (bytes + offsets), custkeys, customer keys."""
    _fields_ = [("o_comment", C.c_void_p), ("o_comment_offsets", C.c_void_p), ("o_custkey", C.c_void_p),
                ("n_orders", C.c_int64), ("c_custkey", C.c_void_p), ("n_customer", C.c_int64),
                ("n_count_map", C.c_int64)]


class TpchQ13Row(C.Structure):
    _fields_ = [("c_count", C.c_int64), ("custdist", C.c_int64)]


BATCH_SCAN_AGG, BATCH_JOIN, BATCH_GROUPBY = 0, 1, 2
BATCH_MAX_CATS = 64


class BatchInstance(C.Structure):
    """``bo_batch_instance``: one pipeline of a batch (fields per kind)."""
    _fields_ = [("kind", C.c_int32), ("tile_rows", C.c_int32), ("predicted", C.c_float),
                ("presize_factor", C.c_float), ("fact", FactCols), ("ship_cutoff", C.c_int32),
                ("n_flag_a", C.c_int32), ("n_flag_b", C.c_int32), ("pad0", C.c_int32),
                ("build", JoinBuildCols), ("probe", JoinProbeCols), ("join", JoinParams),
                ("a", GbACols), ("b", GbBCols), ("c", GbCCols), ("categories", C.c_uint16 * BATCH_MAX_CATS),
                ("n_categories", C.c_int32), ("year_lo", C.c_int32), ("year_hi", C.c_int32), ("k", C.c_int32),
                ("a_id_max", C.c_int32), ("pad1", C.c_int32), ("predicted_device", C.c_void_p)]


class BatchResult(C.Structure):
    _fields_ = [("kind", C.c_int32), ("overflowed", C.c_int32), ("reruns", C.c_int32), ("pad", C.c_int32),
                ("q1", Q1Agg * Q1_MAX_GROUPS), ("join", JoinResult), ("groupby", GbResult)]


SKETCH_BINS = 64


class Sketch(C.Structure):
    _fields_ = [("n", C.c_int64), ("min", C.c_int64), ("max", C.c_int64), ("hist", C.c_int64 * SKETCH_BINS),
                ("distinct_estimate", C.c_double)]


# --------------------------------------------------------------- prototypes --
_P = C.c_void_p
_SIGNATURES = {
    "bo_create": (C.c_int, [C.POINTER(_P), C.c_int]),
    "bo_device_init": (C.c_int, [C.c_int]),
    "bo_destroy": (None, [_P]),
    "bo_last_error": (C.c_char_p, [_P]),
    "bo_set_stream": (C.c_int, [_P, _P]),
    "bo_get_stream": (_P, [_P]),
    "bo_synchronize": (C.c_int, [_P]),
    "bo_num_sms": (C.c_int, [_P]),
    "bo_build_info": (C.c_char_p, []),
    "bo_device_alloc": (C.c_int, [_P, C.c_size_t, C.POINTER(_P)]),
    "bo_device_free": (C.c_int, [_P, _P]),
    "bo_host_alloc_pinned": (C.c_int, [_P, C.c_size_t, C.POINTER(_P)]),
    "bo_host_free_pinned": (C.c_int, [_P, _P]),
    "bo_copy_h2d": (C.c_int, [_P, _P, _P, C.c_size_t]),
    "bo_copy_d2h": (C.c_int, [_P, _P, _P, C.c_size_t]),
    "bo_launch_count": (C.c_int64, [_P]),
    "bo_check_errors": (C.c_int, [_P]),
    "bo_q1_fact_device": (C.c_int, [_P, C.POINTER(FactCols), C.c_int32, C.c_int32, C.c_int32, _P]),
    "bo_q1_fact_host": (C.c_int, [_P, C.POINTER(FactCols), C.c_int32, C.c_int32, C.c_int32, C.POINTER(Q1Agg)]),
    "bo_q1_fact_device_noalloc": (C.c_int, [C.POINTER(FactCols), C.c_int32, C.c_int32, C.c_int32, _P, _P, _P]),
    "bo_q1_lineitem_device": (C.c_int, [_P, C.POINTER(LineitemCols), C.c_int16, C.c_int32, _P]),
    "bo_q1_lineitem_host": (C.c_int, [_P, C.POINTER(LineitemCols), C.c_int16, C.c_int32, C.POINTER(Q1Agg)]),
    "bo_q6_lineitem_device": (
        C.c_int, [_P, C.POINTER(LineitemCols), C.c_int16, C.c_int16, C.c_int32, C.c_int32, C.c_int32, _P]),
    "bo_q6_lineitem_host": (
        C.c_int,
        [_P, C.POINTER(LineitemCols), C.c_int16, C.c_int16, C.c_int32, C.c_int32, C.c_int32, C.POINTER(Q6Result)]),
    "bo_join_count_device": (C.c_int, [_P, C.POINTER(JoinBuildCols), C.POINTER(JoinParams), _P]),
    "bo_join_plain": (C.c_int, [_P, C.POINTER(JoinBuildCols), C.POINTER(JoinProbeCols), C.POINTER(JoinParams),
                                C.POINTER(JoinResult)]),
    "bo_join_presized_device": (C.c_int, [_P, C.POINTER(JoinBuildCols), C.POINTER(JoinProbeCols),
                                          C.POINTER(JoinParams), _P, _P]),
    "bo_join_presized": (C.c_int, [_P, C.POINTER(JoinBuildCols), C.POINTER(JoinProbeCols), C.POINTER(JoinParams),
                                   _P, C.POINTER(JoinResult)]),
    "bo_groupby_topk_plain": (C.c_int, [_P, C.POINTER(GbACols), C.POINTER(GbBCols), C.POINTER(GbCCols),
                                         C.POINTER(GbParams), C.POINTER(GbResult)]),
    "bo_groupby_topk_presized_device": (C.c_int, [_P, C.POINTER(GbACols), C.POINTER(GbBCols), C.POINTER(GbCCols),
                                                   C.POINTER(GbParams), _P, _P]),
    "bo_groupby_topk_presized": (C.c_int, [_P, C.POINTER(GbACols), C.POINTER(GbBCols), C.POINTER(GbCCols),
                                            C.POINTER(GbParams), _P, C.POINTER(GbResult)]),
    "bo_groupby_distinct_device": (C.c_int, [_P, C.POINTER(GbACols), C.POINTER(GbBCols), C.POINTER(GbCCols),
                                              C.POINTER(GbParams), _P]),
    "bo_groupby_a_mask_device": (C.c_int, [_P, C.POINTER(GbACols), C.c_int32, _P]),
    "bo_radix_sort_pairs_device": (C.c_int, [_P, _P, _P, C.c_int64, C.c_int32, C.c_int32]),
    "bo_radix_sort_pairs_host": (C.c_int, [_P, _P, _P, C.c_int64, C.c_int32, C.c_int32]),
    "bo_sketch_i32": (C.c_int, [_P, _P, C.c_int64, C.POINTER(Sketch)]),
    "bo_histogram_small": (C.c_int, [_P, _P, C.c_int32, C.c_int64, C.c_int32, _P]),
    "bo_mlp_create": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_uint64, C.POINTER(_P)]),
    "bo_mlp_destroy": (None, [_P]),
    "bo_mlp_num_params": (C.c_int32, [_P]),
    "bo_mlp_get_params": (C.c_int, [_P, _P, _P]),
    "bo_mlp_set_params": (C.c_int, [_P, _P, _P]),
    "bo_mlp_gradients_device": (C.c_int, [_P, _P, _P, _P, C.c_int32, _P, _P]),
    "bo_mlp_train_step_device": (C.c_int, [_P, _P, _P, _P, C.c_int32, C.c_float, _P]),
    "bo_mlp_train_host": (C.c_int, [_P, _P, _P, _P, C.c_int32, C.c_int32, C.c_float, C.POINTER(C.c_float)]),
    "bo_mlp_infer_device": (C.c_int, [_P, _P, _P, C.c_int32, _P]),
    "bo_mlp_predict_counts": (C.c_int, [_P, _P, _P, _P, _P]),
    "bo_tpch_q3": (C.c_int, [_P, C.POINTER(TpchQ3Tables), C.c_int16, C.c_int32, C.POINTER(TpchQ3Row), C.c_int64,
                             C.POINTER(C.c_int64)]),
    "bo_tpch_order_ranges": (C.c_int, [_P, _P, C.c_int64, _P, C.c_int64, C.c_int64, _P, _P]),
    "bo_tpch_q10": (C.c_int, [_P, C.POINTER(TpchQ10Tables), C.c_int16, C.c_int16, C.c_int32, C.c_int32,
                              C.POINTER(TpchQ10Row), C.c_int64, C.POINTER(C.c_int64)]),
    "bo_tpch_q4": (C.c_int, [_P, C.POINTER(TpchQ4Tables), C.c_int16, C.c_int16, C.POINTER(C.c_int64)]),
    "bo_tpch_q5": (C.c_int, [_P, C.POINTER(TpchQ5Tables), C.c_char_p, C.c_int16, C.c_int16, C.POINTER(C.c_int64)]),
    "bo_tpch_q7": (C.c_int, [_P, C.POINTER(TpchQ7Tables), C.c_char_p, C.c_int64, C.c_int32, C.c_int32, C.c_int16,
                             C.c_int16, C.c_int16, C.POINTER(C.c_int64)]),
    "bo_tpch_q8": (C.c_int, [_P, C.POINTER(TpchQ8Tables), C.c_char_p, C.c_int32, C.c_char_p, C.c_int64, C.c_int32,
                             C.c_int16, C.c_int16, C.c_int16, C.POINTER(C.c_int64)]),
    "bo_tpch_q22": (C.c_int, [_P, C.POINTER(TpchQ22Tables), C.c_char_p, C.c_void_p, C.c_int32,
                              C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "bo_tpch_q11": (C.c_int, [_P, C.POINTER(TpchQ11Tables), C.c_char_p, C.c_int64, C.POINTER(C.c_int64),
                              C.POINTER(C.c_int64)]),
    "bo_tpch_q15": (C.c_int, [_P, C.POINTER(TpchQ15Tables), C.c_int64, C.c_int16, C.c_int16, C.POINTER(C.c_int64),
                              C.POINTER(C.c_int64)]),
    "bo_tpch_q17": (C.c_int, [_P, C.POINTER(TpchQ17Tables), C.c_int32, C.c_int32, C.POINTER(C.c_int64)]),
    "bo_tpch_q19": (C.c_int, [_P, C.POINTER(TpchQ19Tables), C.POINTER(C.c_int32), _P, C.c_int32,
                              C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.c_int32, C.c_int32, C.c_int32,
                              C.POINTER(C.c_int64)]),
    "bo_tpch_q21": (C.c_int, [_P, C.POINTER(TpchQ21Tables), C.c_int32, _P, C.c_int32, _P]),
    "bo_ceb_q3b": (C.c_int, [_P, C.POINTER(CebQ3bTables), C.POINTER(CebQ3bParams), _P, C.c_int64,
                             C.POINTER(C.c_int64)]),
    "bo_ceb_q10a": (C.c_int, [_P, C.POINTER(CebQ10aTables), C.POINTER(CebQ10aParams), _P, C.c_int64,
                              C.POINTER(C.c_int64), C.POINTER(C.c_int32)]),
    "bo_ceb_sort_rows": (C.c_int, [_P, _P, _P, C.c_int64, _P]),
    "bo_ceb_gather_i32": (C.c_int, [_P, _P, _P, C.c_int64, _P]),
    "bo_ceb_gather_u8": (C.c_int, [_P, _P, _P, C.c_int64, _P]),
    "bo_ceb_q1a": (C.c_int, [_P, C.POINTER(CebQ1aTables), C.POINTER(CebQ1aParams), C.POINTER(C.c_int64)]),
    "bo_tpch_q9": (C.c_int, [_P, C.POINTER(TpchQ9Tables), C.c_char_p, C.c_int32, C.c_int32, C.c_int32, _P, _P]),
    "bo_tpch_order_years": (C.c_int, [_P, _P, C.c_int64, _P, C.c_int64, C.c_int16, _P, C.c_int32, C.c_int32, _P]),
    "bo_tpch_q14": (C.c_int, [_P, C.POINTER(TpchQ14Tables), C.c_int16, C.c_int16, C.POINTER(C.c_int64)]),
    "bo_tpch_q12": (C.c_int, [_P, C.POINTER(TpchQ12Tables), C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int16,
                              C.c_int16, C.POINTER(C.c_int64)]),
    "bo_tpch_supplier_complaints": (C.c_int, [_P, _P, _P, _P, C.c_int64, _P, C.c_int64]),
    "bo_tpch_q16": (C.c_int, [_P, C.POINTER(TpchQ16Tables), C.POINTER(TpchQ16Params), C.POINTER(TpchQ16Row),
                              C.c_int64, C.POINTER(C.c_int64)]),
    "bo_tpch_q20": (C.c_int, [_P, C.POINTER(TpchQ20Tables), C.c_char_p, C.c_int32, C.c_int32, C.c_int16,
                              C.c_int16, _P, C.c_int64, C.POINTER(C.c_int64)]),
    "bo_tpch_q2": (C.c_int, [_P, C.POINTER(TpchQ2Tables), C.c_int32, _P, C.c_int32, _P, C.c_int32,
                             C.POINTER(TpchQ2Row), C.c_int64, C.POINTER(C.c_int64)]),
    "bo_tpch_q11_rows": (C.c_int, [_P, C.POINTER(TpchQ11Tables), C.c_char_p, C.c_int64, C.c_double,
                                   C.POINTER(TpchQ11Row), C.c_int64, C.POINTER(C.c_int64)]),
    "bo_tpch_q10_host_rows": (C.c_int, [_P, C.POINTER(TpchQ10Tables), C.c_int16, C.c_int16, C.c_int32, C.c_int32,
                                        C.POINTER(TpchQ10HostStrings), _P, C.c_int64, C.POINTER(C.c_int64)]),
    "bo_tpch_q13": (C.c_int, [_P, C.POINTER(TpchQ13Tables), C.c_char_p, C.c_int64, C.c_char_p, C.c_int64,
                              C.POINTER(TpchQ13Row), C.c_int64, C.POINTER(C.c_int64)]),
    "bo_tpch_q18": (C.c_int, [_P, C.POINTER(TpchQ18Tables), C.c_int32, C.POINTER(TpchQ18Row), C.c_int64,
                              C.POINTER(C.c_int64)]),
    "bo_batch_create": (C.c_int, [_P, C.POINTER(BatchInstance), C.c_int32, C.c_int32, C.POINTER(_P)]),
    "bo_batch_create_pool": (C.c_int, [_P, C.c_int32, C.c_int64, C.c_int64, C.c_int32, C.POINTER(_P)]),
    "bo_batch_update": (C.c_int, [_P, _P, C.POINTER(BatchInstance), C.c_int32]),
    "bo_batch_footprint": (C.c_int, [C.POINTER(BatchInstance), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "bo_batch_launch": (C.c_int, [_P, _P]),
    "bo_batch_results": (C.c_int, [_P, _P, C.POINTER(BatchResult)]),
    "bo_batch_last_ms": (C.c_float, [_P]),
    "bo_batch_done": (C.c_int, [_P]),
    "bo_batch_num_items": (C.c_int32, [_P]),
    "bo_batch_destroy": (None, [_P]),
    "bo_join_probe_device": (C.c_int, [_P, C.POINTER(JoinProbeCols), _P]),
    "bo_join_stream_host": (C.c_int, [_P, C.POINTER(JoinBuildCols), C.POINTER(JoinProbeCols), C.POINTER(JoinParams),
                                      _P, C.POINTER(JoinResult)]),
    "bo_join_stream_host_async": (C.c_int, [_P, C.POINTER(JoinBuildCols), C.POINTER(JoinProbeCols),
                                            C.POINTER(JoinParams), _P, _P]),
    "bo_set_host_threads": (C.c_int, [_P, C.c_int32]),
    "bo_host_threads": (C.c_int, [_P]),
    "bo_groupby_topk_partitioned_device": (C.c_int, [_P, C.POINTER(GbACols), C.POINTER(GbBCols), C.POINTER(GbCCols),
                                                     C.POINTER(GbParams), C.c_int32, C.c_float, _P]),
    "bo_groupby_topk_partitioned": (C.c_int, [_P, C.POINTER(GbACols), C.POINTER(GbBCols), C.POINTER(GbCCols),
                                              C.POINTER(GbParams), C.c_int32, C.c_float, C.POINTER(GbResult)]),
    "bo_join_learned_device": (C.c_int, [_P, _P, _P, C.POINTER(JoinBuildCols), C.POINTER(JoinProbeCols),
                                         C.POINTER(JoinParams), _P, _P]),
    "bo_join_learned": (C.c_int, [_P, _P, _P, C.POINTER(JoinBuildCols), C.POINTER(JoinProbeCols),
                                  C.POINTER(JoinParams), C.POINTER(JoinResult)]),
    "bo_join_partitioned_device": (C.c_int, [_P, C.POINTER(JoinBuildCols), C.POINTER(JoinProbeCols),
                                             C.POINTER(JoinParams), C.c_int32, _P]),
    "bo_join_partitioned": (C.c_int, [_P, C.POINTER(JoinBuildCols), C.POINTER(JoinProbeCols), C.POINTER(JoinParams),
                                      C.c_int32, C.POINTER(JoinResult)]),
    "bo_join_multi_device": (C.c_int, [_P, C.POINTER(JoinBuildCols), C.POINTER(JoinProbeCols), C.POINTER(JoinParams),
                                       C.c_int32, _P]),
    "bo_join_multi_host": (C.c_int, [_P, C.POINTER(JoinBuildCols), C.POINTER(JoinProbeCols), C.POINTER(JoinParams),
                                     C.c_int32, C.POINTER(JoinResult)]),
    "bo_join_host": (C.c_int, [_P, C.POINTER(JoinBuildCols), C.POINTER(JoinProbeCols), C.POINTER(JoinParams),
                               C.c_int32, C.c_float, C.POINTER(JoinResult)]),
}

_lib = None
_lib_lock = threading.Lock()


def register(name: str, restype, argtypes) -> None:
    """Adds a prototype (used by the modules that bind later entry points)."""
    _SIGNATURES[name] = (restype, argtypes)
    if _lib is not None:
        f = getattr(_lib, name)
        f.restype, f.argtypes = restype, argtypes


def lib() -> C.CDLL:
    """Loads the engine library; raises if it has not been built."""
    global _lib
    with _lib_lock:
        if _lib is None:
            if not LIB_PATH.exists():
                raise RuntimeError(
                    f"{LIB_PATH} is missing: build it with `python -m bespokeolap_artifacts_b200.build` "
                    "(the engine has no CPU fallback)")
            l = C.CDLL(str(LIB_PATH))
            for name, (res, args) in _SIGNATURES.items():
                f = getattr(l, name)
                f.restype, f.argtypes = res, args
            _lib = l
    return _lib


def ptr(a) -> int:
    """Raw address of a numpy array or torch tensor (host or device)."""
    if a is None:
        return 0
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    if isinstance(a, int):
        return a
    raise TypeError(f"cannot take the address of {type(a)}")


class Context:
    """Owns one ``bo_ctx`` (one CUDA stream and its scratch state)."""

    def __init__(self, device: int = 0):
        self._lib = lib()
        h = C.c_void_p()
        rc = self._lib.bo_create(C.byref(h), device)
        if rc != BO_OK:
            raise BoError(rc, f"bo_create(device={device}) failed (no sm_100 GPU visible?)")
        self.handle = h
        self.device = device

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.bo_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def check(self, rc: int, what: str = "") -> None:
        if rc != BO_OK:
            msg = self._lib.bo_last_error(self.handle)
            raise BoError(rc, f"{what}: {msg.decode() if msg else ''}")

    def call(self, name: str, *args) -> None:
        self.check(getattr(self._lib, name)(self.handle, *args), name)

    @property
    def num_sms(self) -> int:
        return self._lib.bo_num_sms(self.handle)

    @property
    def launches(self) -> int:
        return self._lib.bo_launch_count(self.handle)

    def set_stream(self, stream_handle: int | None) -> None:
        self.call("bo_set_stream", C.c_void_p(stream_handle or 0))

    def synchronize(self) -> None:
        self.call("bo_synchronize")
