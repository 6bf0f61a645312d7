// Drop-in GPU host for the reference's TPC-H engine.
//
// The reference's external driver links three C++ entry points
// (bespoke_tpch/loader_impl.hpp:20, builder_impl.hpp:173, query_impl.hpp:6):
//     ParquetTables* load(std::string);   Database* build(ParquetTables*);   void query(Database*);
// This library exports the same three signatures, so that driver links
// unchanged.  load() reads the same eight Parquet files; build() derives the
// storage-plan columns the hot path reads (the reference builder's rules,
// bespoke_tpch/builder_impl.cpp:447-999, restated) and uploads them once;
// query() speaks the same stdin / result<idx>.csv / "Execution ms" protocol
// (bespoke_tpch/query_impl.cpp:142-389) and runs Q1, Q3, Q6, Q10, Q13 and Q18
// on the GPU through the C ABI of include/bespoke_gpu.h.  Result structs and
// CSV formats are the reference's (query_q1.hpp:9-20, query_q3.hpp:10-15,
// query_q6.hpp, query_q10.hpp:10-19, query_q13.hpp:9-12, query_q18.hpp:10-17).
// Requests for other query ids get the reference's stub CSV
// (query_impl.cpp:98-103): this library has no CPU implementation of them.
#pragma once

#include <arrow/table.h>

#include <cstdint>
#include <memory>
#include <string>
#include <unordered_map>
#include <utility>
#include <string_view>
#include <vector>

#include "bespoke_gpu.h"

struct ParquetTables {
  using ArrowTable = std::shared_ptr<arrow::Table>;

  ArrowTable customer;
  ArrowTable lineitem;
  ArrowTable nation;
  ArrowTable orders;
  ArrowTable part;
  ArrowTable partsupp;
  ArrowTable region;
  ArrowTable supplier;
};

namespace bo_tpch {

// One device allocation per column, freed with the database.
struct DeviceColumn {
  void* ptr = nullptr;
  int64_t rows = 0;
};

struct Dictionary {
  std::vector<std::string> values;  // first-appearance order
};

// Host strings the result rows carry: values concatenated, row i at
// [offsets[i], offsets[i + 1]) (bespoke_tpch/builder_impl.hpp StringColumn).
struct StringColumn {
  std::string data;
  std::vector<uint32_t> offsets;
  std::string_view view(size_t row) const {
    return std::string_view(data.data() + offsets[row], offsets[row + 1] - offsets[row]);
  }
};

}  // namespace bo_tpch

// GPU-resident database: the storage-plan columns the GPU queries read, on
// the device; dictionaries, sizes and the strings of result rows on the host.
struct Database {
  int32_t base_date_days = 0;
  bo_ctx* ctx = nullptr;
  // lineitem (row order of the input)
  int64_t n_lineitem = 0;
  bo_tpch::DeviceColumn l_orderkey, l_shipdate, l_returnflag_linestatus, l_extendedprice, l_discounted_price,
      l_discount, l_tax, l_quantity, l_shipmode, l_commit_receipt, l_partkey, l_supp_nation, l_suppkey;
  // Latest shipdate of each lineitem's builder shard; only built when some
  // lineitem is received more than 30 days after shipping (Q12's shard pruning).
  bo_tpch::DeviceColumn l_shard_max_shipdate;
  bo_tpch::Dictionary returnflag, linestatus, shipmode, shipinstruct;
  bo_tpch::DeviceColumn l_shipinstruct;  // dictionary codes (Q19)
  int32_t max_lineitem_partkey = -1;
  bool lineitem_orderkey_sorted = true;
  int32_t max_lineitem_orderkey = -1;
  // orders, sorted by orderdate (stable); each row's lineitem range
  int64_t n_orders = 0;
  bo_tpch::DeviceColumn o_orderkey, o_custkey, o_orderdate, o_shippriority, o_totalprice, orderkey_to_row,
      o_li_begin, o_li_end, o_comment, o_comment_offsets, o_orderpriority, o_cust_nation;
  bo_tpch::Dictionary orderpriority, orderstatus;
  bo_tpch::DeviceColumn o_orderstatus;  // dictionary codes (Q21)
  int64_t n_orderkey_map = 0;
  bool dense_orderkeys = false;  // first orderkey 1, last n_orders (date order)
  // customer; custkey_to_row keeps the last row of each custkey >= 0
  int64_t n_customer = 0;
  int32_t custkey_bound = 0;
  bool dense_custkeys = false;  // first custkey 1, last n_customer
  bo_tpch::DeviceColumn c_custkey, c_mktsegment, c_nationkey, custkey_to_row;
  int64_t n_custkey_map = 0;
  bo_tpch::Dictionary mktsegment;
  std::vector<int32_t> c_acctbal;
  // Q22: balances on the device, phone classes (numeric two-digit prefix or
  // 255; 0x10000 | first two bytes for phones of two bytes or more), and a
  // bit per custkey that has an order (custkeys 0 .. largest order custkey)
  bo_tpch::DeviceColumn c_acctbal_device, c_phone_prefix, c_phone_pair, o_has_order;
  int64_t n_order_custkeys = 0;
  bo_tpch::StringColumn c_name, c_address, c_phone, c_comment;
  // their offsets on the device (Q10 result rows carry each customer's ranges)
  bo_tpch::DeviceColumn c_name_offsets, c_address_offsets, c_phone_offsets, c_comment_offsets;
  // part: per partkey 1 (PROMO type), 0 (other type), -1 (no part row); the
  // largest partkey (-1 without parts)
  bo_tpch::DeviceColumn p_promo_by_key;
  int64_t n_promo_map = 0;
  int32_t max_partkey = -1;
  // part rows: keys, brand and container codes (Q17); names as bytes with
  // n_part + 1 offsets (Q9's color search on the device)
  bo_tpch::DeviceColumn p_partkey, p_brand, p_container, p_type, p_name, p_name_offsets;
  // part sizes and the last part row of each key 0 .. max_partkey, -1 = none (Q19)
  bo_tpch::DeviceColumn p_size, p_row_by_key;
  int64_t n_part = 0;
  bo_tpch::Dictionary brand, container, part_type;
  // nation names by nationkey in [0, nation_bound) (last row of each key)
  int32_t nation_bound = 1;
  std::vector<std::string> nation_name;
  std::vector<bo_host_str> nation_name_str;  // the same names as host strings (Q10's rows point at them)
  // nation rows' keys, region keys and names; region name -> key (first row of a name)
  std::vector<int32_t> nation_key, nation_regionkey;
  std::vector<std::string> nation_row_name;
  // partsupp sorted by partkey (stable), value = supplycost * availqty (x100)
  bo_tpch::DeviceColumn ps_partkey, ps_suppkey, ps_value;
  int64_t n_partsupp = 0;
  // Q9: supplycost (x100) in the same order; each partkey's rows
  // [ps_part_begin[k], ps_part_begin[k + 1]) for k in [0, n_ps_part_keys)
  // (the largest part / partsupp key + 1, query_q9.cpp:140-141) and the
  // largest row count of a key (the reference's slots per part)
  bo_tpch::DeviceColumn ps_supplycost, ps_part_begin;
  int64_t n_ps_part_keys = 0;
  int32_t ps_slots_per_part = 1;
  // orders' first and last date offsets; Q9's per-orderkey year table
  // (filled per query, n_orderkey_map entries)
  int16_t o_min_date = 0, o_max_date = -1;
  bo_tpch::DeviceColumn o_year_by_key;
  int32_t ps_min_partkey = 0, ps_max_partkey = -1;
  // supplier rows' keys and nationkeys (Q7's supplier tags), strings (Q15)
  std::vector<int32_t> s_suppkey, s_nationkey;
  bo_tpch::StringColumn s_name, s_address, s_phone;
  // Supplier comments and, by suppkey, run_q16's complaint flags (computed on
  // the device at build: they do not depend on a query's parameters).
  bo_tpch::StringColumn s_comment;
  bo_tpch::DeviceColumn s_comment_chars, s_comment_offsets, s_suppkey_device, s_banned;
  int64_t n_s_banned = 0;
  // Ranks of the brand and type dictionary entries in string order (Q16's tie order).
  std::vector<uint16_t> brand_rank, type_rank;
  // Q20: supplier nations by suppkey (-1: none), nations and rows in s_name order.
  bo_tpch::DeviceColumn s_nation_by_key, s_nationkey_device, s_row_by_name, ps_availqty;
  int32_t s_max_suppkey = -1;
  // Q2: balances (x100), nation index by supplier row (the nation key when below
  // the nation row count, else -1) with its name, and each row's position in
  // (acctbal desc, nation name, s_name, row) order.
  std::vector<int32_t> s_acctbal, s_nation_idx;
  std::vector<std::string> nation_name_by_idx;
  bo_tpch::DeviceColumn s_nation_idx_device, s_rank, p_mfgr;
  bo_tpch::Dictionary mfgr;
  std::unordered_map<std::string, int32_t> region_key_by_name;
  // Result record of the last scan-agg / Q6 query.  Queries on one Database
  // run one at a time (as the reference's single-threaded query()).
  bo_tpch::DeviceColumn scratch;
  // Pinned host buffer the multi-row queries receive their records in; grown
  // on demand, never cleared (each call reads only the rows it was given).
  mutable void* result_host = nullptr;
  mutable size_t result_host_bytes = 0;
  ~Database();
};

ParquetTables* load(std::string);
Database* build(ParquetTables*);
void query(Database*);

// ---------------------------------------------------------------- queries --
struct Q1ResultRow {
  std::string returnflag;
  std::string linestatus;
  double sum_qty = 0.0;
  double sum_base_price = 0.0;
  double sum_disc_price = 0.0;
  double sum_charge = 0.0;
  double avg_qty = 0.0;
  double avg_price = 0.0;
  double avg_disc = 0.0;
  int64_t count_order = 0;
};

// Q3ResultRow (bespoke_tpch/query_q3.hpp:10-15) as the GPU writes it.
using Q3ResultRow = bo_tpch_q3_row;

struct Q6ResultRow {
  int64_t revenue_raw = 0;
};

struct Q4ResultRow {
  std::string orderpriority;
  int64_t order_count = 0;
};

struct Q5ResultRow {
  std::string n_name;
  int64_t revenue_raw = 0;
};

struct Q7ResultRow {
  std::string supp_nation;
  std::string cust_nation;
  int32_t l_year = 0;
  int64_t revenue_raw = 0;
};

struct Q8ResultRow {
  int32_t o_year = 0;
  double mkt_share = 0.0;
};

struct Q22ResultRow {
  std::string cntrycode;
  int64_t numcust = 0;
  int64_t totacctbal_raw = 0;
};

struct Q9ResultRow {
  std::string nation;
  int32_t o_year = 0;
  int64_t sum_profit_raw = 0;
};

struct Q19ResultRow {
  int64_t revenue_raw = 0;
};

struct Q21ResultRow {
  std::string_view s_name;
  int64_t numwait = 0;
};

struct Q11ResultRow {
  int32_t ps_partkey = 0;
  int64_t value_raw = 0;
};

struct Q15ResultRow {
  int32_t s_suppkey = 0;
  std::string_view s_name, s_address, s_phone;
  int64_t total_revenue_raw = 0;
};

struct Q17ResultRow {
  int64_t sum_extendedprice_raw = 0;
};

struct Q14ResultRow {
  double promo_revenue = 0.0;
};

struct Q12ResultRow {
  std::string shipmode;
  int64_t high_line_count = 0;
  int64_t low_line_count = 0;
};

struct Q13ResultRow {
  int64_t c_count = 0;
  int64_t custdist = 0;
};

struct Q20ResultRow {
  std::string_view s_name;
  std::string_view s_address;
};

struct Q2ResultRow {
  int32_t s_acctbal_raw = 0;
  std::string_view s_name;
  std::string_view n_name;
  int32_t p_partkey = 0;
  std::string_view p_mfgr;
  std::string_view s_address;
  std::string_view s_phone;
  std::string_view s_comment;
};

struct Q16ResultRow {
  std::string_view p_brand;
  std::string_view p_type;
  int32_t p_size = 0;
  int64_t supplier_cnt = 0;
};

// Q10ResultRow (bespoke_tpch/query_q10.hpp:10-19) as the GPU writes it into
// the Database's mapped pinned result buffer: the strings are host pointers
// into the Database's customer columns and nation names.
using Q10ResultRow = bo_tpch_q10_host_row;
inline std::string_view view_of(const bo_host_str& s) { return std::string_view(s.ptr, s.len); }

// The rows of one request as the GPU left them in the Database's pinned
// result buffer: a view, valid until the Database answers its next query.
template <class Row>
class RowView {
 public:
  RowView() = default;
  RowView(const Row* rows, size_t n) : rows_(rows), n_(n) {}
  const Row* begin() const { return rows_; }
  const Row* end() const { return rows_ + n_; }
  size_t size() const { return n_; }
  bool empty() const { return n_ == 0; }
  const Row& operator[](size_t i) const { return rows_[i]; }

 private:
  const Row* rows_ = nullptr;
  size_t n_ = 0;
};
using Q10Rows = RowView<Q10ResultRow>;

struct Q18ResultRow {
  std::string_view c_name;
  int32_t c_custkey = 0;
  int32_t o_orderkey = 0;
  int16_t o_orderdate_offset = 0;
  int32_t o_totalprice_raw = 0;
  int64_t sum_qty_raw = 0;
};

namespace bo_tpch {

int64_t days_from_civil(int64_t y, unsigned m, unsigned d);
void civil_from_days(int64_t z, int& y, unsigned& m, unsigned& d);

// Run on the GPU; the arguments are the request's strings (DELTA; SEGMENT,
// DATE; DATE, DISCOUNT, QUANTITY; DATE; WORD1, WORD2; QUANTITY), parsed as the
// reference parses them.
std::vector<Q1ResultRow> run_q1(const Database& db, const std::string& delta);
RowView<Q3ResultRow> run_q3(const Database& db, const std::string& segment, const std::string& date);
std::vector<Q6ResultRow> run_q6(const Database& db, const std::string& date, const std::string& discount,
                                const std::string& quantity);
Q10Rows run_q10(const Database& db, const std::string& date);
std::vector<Q4ResultRow> run_q4(const Database& db, const std::string& date);
std::vector<Q5ResultRow> run_q5(const Database& db, const std::string& region, const std::string& date);
std::vector<Q7ResultRow> run_q7(const Database& db, const std::string& nation1, const std::string& nation2);
std::vector<Q8ResultRow> run_q8(const Database& db, const std::string& nation, const std::string& region,
                                const std::string& type);
std::vector<Q22ResultRow> run_q22(const Database& db, const std::vector<std::string>& codes);
std::vector<Q11ResultRow> run_q11(const Database& db, const std::string& nation, const std::string& fraction);
std::vector<Q15ResultRow> run_q15(const Database& db, const std::string& date);
std::vector<Q9ResultRow> run_q9(const Database& db, const std::string& color);
std::vector<Q21ResultRow> run_q21(const Database& db, const std::string& nation);
std::vector<Q19ResultRow> run_q19(const Database& db, const std::string quantity[3], const std::string brand[3]);
std::vector<Q17ResultRow> run_q17(const Database& db, const std::string& brand, const std::string& container);
std::vector<Q14ResultRow> run_q14(const Database& db, const std::string& date);
std::vector<Q12ResultRow> run_q12(const Database& db, const std::string& shipmode1, const std::string& shipmode2,
                                  const std::string& date);
std::vector<Q13ResultRow> run_q13(const Database& db, const std::string& word1, const std::string& word2);
std::vector<Q18ResultRow> run_q18(const Database& db, const std::string& quantity);
std::vector<Q16ResultRow> run_q16(const Database& db, const std::string& brand, const std::string& type,
                                  const std::string sizes[8]);

void write_q1_csv(const std::string& filename, const std::vector<Q1ResultRow>& rows);
void write_q3_csv(const Database& db, const std::string& filename, const RowView<Q3ResultRow>& rows);
void write_q6_csv(const std::string& filename, const std::vector<Q6ResultRow>& rows);
void write_q10_csv(const std::string& filename, const Q10Rows& rows);
void write_q4_csv(const std::string& filename, const std::vector<Q4ResultRow>& rows);
void write_q5_csv(const std::string& filename, const std::vector<Q5ResultRow>& rows);
void write_q7_csv(const std::string& filename, const std::vector<Q7ResultRow>& rows);
void write_q8_csv(const std::string& filename, const std::vector<Q8ResultRow>& rows);
void write_q22_csv(const std::string& filename, const std::vector<Q22ResultRow>& rows);
void write_q11_csv(const std::string& filename, const std::vector<Q11ResultRow>& rows);
void write_q15_csv(const std::string& filename, const std::vector<Q15ResultRow>& rows);
void write_q9_csv(const std::string& filename, const std::vector<Q9ResultRow>& rows);
void write_q21_csv(const std::string& filename, const std::vector<Q21ResultRow>& rows);
void write_q19_csv(const std::string& filename, const std::vector<Q19ResultRow>& rows);
void write_q17_csv(const std::string& filename, const std::vector<Q17ResultRow>& rows);
void write_q14_csv(const std::string& filename, const std::vector<Q14ResultRow>& rows);
void write_q12_csv(const std::string& filename, const std::vector<Q12ResultRow>& rows);
void write_q13_csv(const std::string& filename, const std::vector<Q13ResultRow>& rows);
void write_q18_csv(const Database& db, const std::string& filename, const std::vector<Q18ResultRow>& rows);
void write_q16_csv(const std::string& filename, const std::vector<Q16ResultRow>& rows);
std::vector<Q20ResultRow> run_q20(const Database& db, const std::string& color, const std::string& date,
                                  const std::string& nation);
void write_q20_csv(const std::string& filename, const std::vector<Q20ResultRow>& rows);
std::vector<Q2ResultRow> run_q2(const Database& db, const std::string& size, const std::string& type,
                                const std::string& region);
void write_q2_csv(const std::string& filename, const std::vector<Q2ResultRow>& rows);

}  // namespace bo_tpch
