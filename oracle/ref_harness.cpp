// ORACLE -- test infrastructure, not part of the product.
//
// Harness that runs the reference's own TPC-H pipelines, compiled unchanged from
// the reference tree, on seeded in-memory inputs:
//   * query_impl.cpp is included as-is (it textually includes every
//     query_qN.cpp, bespoke_tpch/query_impl.cpp:13-56), giving run_q1 / run_q3 /
//     run_q6 / ... and query();
//   * builder_impl.cpp and loader_impl.cpp are compiled as their own units;
//   * the two helpers the reference includes but does not ship
//     (loader_utils.hpp, cpu_affinity.hpp) come from oracle/ref_stubs.
// Raw columns arrive as plain arrays and are turned into the Arrow tables the
// reference's build() consumes (the role of ParquetTables,
// bespoke_tpch/loader_impl.hpp:6-17), so the reference's own builder derives
// its storage-plan layout exactly as it would from Parquet.
//
// Built only where the reference sources exist, by oracle/build_oracle.py, into
// oracle/_ref/.  The tests use it to pin the C restatement (bo_oracle.c) and the
// GPU results; bench.py's reference arm times run_q1 / run_q3 through it.
#include <arrow/api.h>
#include <arrow/io/file.h>
#include <parquet/arrow/reader.h>

#include <chrono>
#include <cstring>
#include <iostream>
#include <sstream>
#include <thread>

#include "query_impl.cpp"

std::shared_ptr<arrow::Table> ReadParquetTable(const std::string& path) {
  auto infile = arrow::io::ReadableFile::Open(path);
  if (!infile.ok()) throw std::runtime_error("cannot open " + path);
  auto reader = parquet::arrow::OpenFile(*infile, arrow::default_memory_pool());
  if (!reader.ok()) throw std::runtime_error("cannot read parquet " + path);
  std::shared_ptr<arrow::Table> table;
  auto st = (*reader)->ReadTable(&table);
  if (!st.ok()) throw std::runtime_error("cannot read table " + path);
  return table;
}

namespace {

template <class Builder, class T>
std::shared_ptr<arrow::Array> make_array(const T* v, int64_t n, T fill) {
  Builder b;
  if (!b.Reserve(n).ok()) throw std::runtime_error("arrow reserve");
  for (int64_t i = 0; i < n; ++i) b.UnsafeAppend(v ? v[i] : fill);
  std::shared_ptr<arrow::Array> out;
  if (!b.Finish(&out).ok()) throw std::runtime_error("arrow finish");
  return out;
}

std::shared_ptr<arrow::Array> i32(const int32_t* v, int64_t n, int32_t fill = 0) {
  return make_array<arrow::Int32Builder>(v, n, fill);
}
std::shared_ptr<arrow::Array> f64(const double* v, int64_t n, double fill = 0.0) {
  return make_array<arrow::DoubleBuilder>(v, n, fill);
}
std::shared_ptr<arrow::Array> date32(const int32_t* v, int64_t n, int32_t fill) {
  return make_array<arrow::Date32Builder>(v, n, fill);
}
std::shared_ptr<arrow::Array> str_const(const char* s, int64_t n) {
  auto r = arrow::MakeArrayFromScalar(arrow::StringScalar(s), n);
  if (!r.ok()) throw std::runtime_error("arrow scalar array");
  return *r;
}
// Strings by code: value = dict[code[i]].
std::shared_ptr<arrow::Array> str_codes(const uint8_t* code, int64_t n, const char* const* dict) {
  if (!code) return str_const(dict[0], n);
  arrow::StringBuilder b;
  if (!b.Reserve(n).ok()) throw std::runtime_error("arrow reserve");
  for (int64_t i = 0; i < n; ++i)
    if (!b.Append(dict[code[i]]).ok()) throw std::runtime_error("arrow append");
  std::shared_ptr<arrow::Array> out;
  if (!b.Finish(&out).ok()) throw std::runtime_error("arrow finish");
  return out;
}

std::shared_ptr<arrow::Table> table(const std::vector<std::pair<std::string, std::shared_ptr<arrow::Array>>>& cols) {
  std::vector<std::shared_ptr<arrow::Field>> fields;
  std::vector<std::shared_ptr<arrow::Array>> arrays;
  for (const auto& c : cols) {
    fields.push_back(arrow::field(c.first, c.second->type()));
    arrays.push_back(c.second);
  }
  return arrow::Table::Make(arrow::schema(fields), arrays);
}

const char* const kFlagA[] = {"A", "B", "C", "D", "E", "F", "G", "H"};
const char* const kFlagB[] = {"V", "W", "X", "Y", "Z"};
const char* const kSegment[] = {"SEG0", "SEG1", "SEG2", "SEG3", "SEG4", "SEG5", "SEG6", "SEG7"};

double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

extern "C" {

// Raw columns of the three TPC-H tables the hot path reads.  Decimal columns are
// given as their decimal values (e.g. 17.5), which build() scales by 100 with
// llround (bespoke_tpch/builder_impl.cpp:70); dates are days since 1970-01-01.
// Null pointers get a constant fill.  Flag codes index kFlagA / kFlagB, segment
// codes index kSegment.
struct ref_tpch_input {
  int64_t n_lineitem;
  const int32_t* l_orderkey;
  const int32_t* l_shipdate;
  const double* l_quantity;
  const double* l_extendedprice;
  const double* l_discount;
  const double* l_tax;
  const uint8_t* l_returnflag;
  const uint8_t* l_linestatus;
  int64_t n_orders;
  const int32_t* o_orderkey;
  const int32_t* o_custkey;
  const int32_t* o_orderdate;
  int64_t n_customer;
  const int32_t* c_custkey;
  const uint8_t* c_mktsegment;
};

struct ref_q1_row {
  char returnflag[8];
  char linestatus[8];
  double sum_qty, sum_base_price, sum_disc_price, sum_charge, avg_qty, avg_price, avg_disc;
  int64_t count_order;
};

// Builds the reference Database through the reference build().  Returns NULL
// and writes a message on failure.
void* ref_tpch_build(const ref_tpch_input* in, double* build_ms, char* err, int err_len) {
  try {
    const int64_t nl = in->n_lineitem, no = in->n_orders, nc = in->n_customer;
    auto* t = new ParquetTables{};
    t->lineitem = table({
        {"l_orderkey", i32(in->l_orderkey, nl, 1)},
        {"l_partkey", i32(nullptr, nl, 1)},
        {"l_suppkey", i32(nullptr, nl, 1)},
        {"l_linenumber", i32(nullptr, nl, 1)},
        {"l_quantity", f64(in->l_quantity, nl)},
        {"l_extendedprice", f64(in->l_extendedprice, nl)},
        {"l_discount", f64(in->l_discount, nl)},
        {"l_tax", f64(in->l_tax, nl)},
        {"l_returnflag", str_codes(in->l_returnflag, nl, kFlagA)},
        {"l_linestatus", str_codes(in->l_linestatus, nl, kFlagB)},
        {"l_shipdate", date32(in->l_shipdate, nl, 8035)},
        {"l_commitdate", date32(nullptr, nl, 8035)},
        {"l_receiptdate", date32(nullptr, nl, 8035)},
        {"l_shipinstruct", str_const("I0", nl)},
        {"l_shipmode", str_const("M0", nl)},
        {"l_comment", str_const("", nl)},
    });
    t->orders = table({
        {"o_orderkey", i32(in->o_orderkey, no, 1)},
        {"o_custkey", i32(in->o_custkey, no, 1)},
        {"o_orderstatus", str_const("S", no)},
        {"o_totalprice", f64(nullptr, no)},
        {"o_orderdate", date32(in->o_orderdate, no, 8035)},
        {"o_orderpriority", str_const("P", no)},
        {"o_clerk", str_const("C", no)},
        {"o_shippriority", i32(nullptr, no, 0)},
        {"o_comment", str_const("", no)},
    });
    t->customer = table({
        {"c_custkey", i32(in->c_custkey, nc, 1)},
        {"c_name", str_const("N", nc)},
        {"c_address", str_const("A", nc)},
        {"c_nationkey", i32(nullptr, nc, 0)},
        {"c_phone", str_const("10-000", nc)},
        {"c_acctbal", f64(nullptr, nc)},
        {"c_mktsegment", str_codes(in->c_mktsegment, nc, kSegment)},
        {"c_comment", str_const("", nc)},
    });
    const int32_t one = 1;
    t->part = table({{"p_partkey", i32(&one, 1)}, {"p_name", str_const("p", 1)}, {"p_mfgr", str_const("m", 1)},
                     {"p_brand", str_const("b", 1)}, {"p_type", str_const("t", 1)}, {"p_size", i32(&one, 1)},
                     {"p_container", str_const("c", 1)}, {"p_retailprice", f64(nullptr, 1)},
                     {"p_comment", str_const("", 1)}});
    t->supplier = table({{"s_suppkey", i32(&one, 1)}, {"s_name", str_const("s", 1)}, {"s_address", str_const("a", 1)},
                         {"s_nationkey", i32(nullptr, 1, 0)}, {"s_phone", str_const("10-0", 1)},
                         {"s_acctbal", f64(nullptr, 1)}, {"s_comment", str_const("", 1)}});
    t->partsupp = table({{"ps_partkey", i32(&one, 1)}, {"ps_suppkey", i32(&one, 1)}, {"ps_availqty", i32(&one, 1)},
                         {"ps_supplycost", f64(nullptr, 1)}, {"ps_comment", str_const("", 1)}});
    t->nation = table({{"n_nationkey", i32(nullptr, 1, 0)}, {"n_name", str_const("NATION0", 1)},
                       {"n_regionkey", i32(nullptr, 1, 0)}, {"n_comment", str_const("", 1)}});
    t->region = table({{"r_regionkey", i32(nullptr, 1, 0)}, {"r_name", str_const("REGION0", 1)},
                       {"r_comment", str_const("", 1)}});
    // build() prints "Build ms"; keep stdout clean for the caller.
    std::ostringstream sink;
    auto* old = std::cout.rdbuf(sink.rdbuf());
    const auto t0 = std::chrono::steady_clock::now();
    Database* db = build(t);
    if (build_ms) *build_ms = ms_since(t0);
    std::cout.rdbuf(old);
    delete t;
    return db;
  } catch (const std::exception& e) {
    if (err && err_len > 0) std::snprintf(err, (size_t)err_len, "%s", e.what());
    return nullptr;
  }
}

void ref_tpch_free(void* db) { delete static_cast<Database*>(db); }

// Storage-plan columns of the built lineitem table (for feeding the GPU the
// exact layout the reference derived).  Pointers stay valid until ref_tpch_free.
struct ref_lineitem_view {
  const int16_t* shipdate;
  const uint8_t* returnflag_linestatus;
  const int32_t* extendedprice;
  const int32_t* discounted_price;
  const uint8_t* discount;
  const uint8_t* tax;
  const int16_t* quantity;
  int64_t n_rows;
  int32_t returnflag_count;
  int32_t linestatus_count;
  int32_t base_date_days;
  int32_t orderkey_sorted;
};

int ref_lineitem(void* dbp, ref_lineitem_view* v, char* rf_dict, char* ls_dict) {
  const Database& db = *static_cast<Database*>(dbp);
  const auto& li = db.lineitem;
  v->shipdate = li.shipdate.data();
  v->returnflag_linestatus = li.returnflag_linestatus.data();
  v->extendedprice = li.extendedprice.data();
  v->discounted_price = li.discounted_price.data();
  v->discount = li.discount.data();
  v->tax = li.tax.data();
  v->quantity = li.quantity.data();
  v->n_rows = (int64_t)li.row_count;
  v->returnflag_count = (int32_t)li.returnflag.dictionary.size();
  v->linestatus_count = (int32_t)li.linestatus.dictionary.size();
  v->base_date_days = db.base_date_days;
  v->orderkey_sorted = li.orderkey_sorted ? 1 : 0;
  // First character of each dictionary entry, in code order.
  for (size_t i = 0; i < li.returnflag.dictionary.size() && i < 15; ++i) rf_dict[i] = li.returnflag.dictionary[i][0];
  for (size_t i = 0; i < li.linestatus.dictionary.size() && i < 15; ++i) ls_dict[i] = li.linestatus.dictionary[i][0];
  return 0;
}

// run_q1 (bespoke_tpch/query_q1.cpp:104) with DELTA = delta_days.
int ref_q1(void* db, int32_t delta_days, ref_q1_row* rows, int max_rows, double* elapsed_ms) {
  Q1Args args;
  args.DELTA = std::to_string(delta_days);
  const auto t0 = std::chrono::steady_clock::now();
  auto out = run_q1(*static_cast<Database*>(db), args);
  if (elapsed_ms) *elapsed_ms = ms_since(t0);
  int n = 0;
  for (const auto& r : out) {
    if (n >= max_rows) break;
    std::snprintf(rows[n].returnflag, 8, "%s", r.returnflag.c_str());
    std::snprintf(rows[n].linestatus, 8, "%s", r.linestatus.c_str());
    rows[n].sum_qty = r.sum_qty;
    rows[n].sum_base_price = r.sum_base_price;
    rows[n].sum_disc_price = r.sum_disc_price;
    rows[n].sum_charge = r.sum_charge;
    rows[n].avg_qty = r.avg_qty;
    rows[n].avg_price = r.avg_price;
    rows[n].avg_disc = r.avg_disc;
    rows[n].count_order = r.count_order;
    ++n;
  }
  return n;
}

// run_q3 (bespoke_tpch/query_q3.cpp:153) with SEGMENT = kSegment[segment],
// DATE = date ("YYYY-MM-DD").  Returns the number of result rows; writes the
// sum of revenue_raw over them and, optionally, the rows themselves.
int64_t ref_q3(void* db, int32_t segment, const char* date, int64_t* revenue_sum, int32_t* orderkeys,
               int64_t* revenues, int64_t max_rows, double* elapsed_ms) {
  Q3Args args;
  args.SEGMENT = kSegment[segment];
  args.DATE = date;
  const auto t0 = std::chrono::steady_clock::now();
  auto out = run_q3(*static_cast<Database*>(db), args);
  if (elapsed_ms) *elapsed_ms = ms_since(t0);
  int64_t s = 0;
  for (size_t i = 0; i < out.size(); ++i) {
    s += out[i].revenue_raw;
    if ((int64_t)i < max_rows) {
      if (orderkeys) orderkeys[i] = out[i].orderkey;
      if (revenues) revenues[i] = out[i].revenue_raw;
    }
  }
  *revenue_sum = s;
  return (int64_t)out.size();
}

// run_q6 (bespoke_tpch/query_q6.cpp:155).
int ref_q6(void* db, const char* date, const char* discount, const char* quantity, int64_t* revenue_raw,
           double* elapsed_ms) {
  Q6Args args;
  args.DATE = date;
  args.DISCOUNT = discount;
  args.QUANTITY = quantity;
  const auto t0 = std::chrono::steady_clock::now();
  auto out = run_q6(*static_cast<Database*>(db), args);
  if (elapsed_ms) *elapsed_ms = ms_since(t0);
  *revenue_raw = out.empty() ? 0 : out[0].revenue_raw;
  return (int)out.size();
}

// run_q18 (bespoke_tpch/query_q18.cpp:183) with QUANTITY = quantity (decimal
// text).  Returns the number of result rows and writes, in the reference's
// output order, each row's orderkey and sum_qty_raw (x100) up to max_rows.
int64_t ref_q18(void* db, const char* quantity, int32_t* orderkeys, int64_t* sum_qty, int64_t max_rows,
                double* elapsed_ms) {
  Q18Args args;
  args.QUANTITY = quantity;
  const auto t0 = std::chrono::steady_clock::now();
  auto out = run_q18(*static_cast<Database*>(db), args);
  if (elapsed_ms) *elapsed_ms = ms_since(t0);
  for (size_t i = 0; i < out.size() && (int64_t)i < max_rows; ++i) {
    if (orderkeys) orderkeys[i] = out[i].o_orderkey;
    if (sum_qty) sum_qty[i] = out[i].sum_qty_raw;
  }
  return (int64_t)out.size();
}

// Runs run_q1 (which != 3) or run_q3 on n_db independent databases, one host
// thread each, and returns the wall time of the slowest: the reference path
// spread over row shards (its sums are decomposable).
double ref_parallel(void** dbs, int n_db, int which, int32_t delta_days, int32_t segment, const char* date,
                    int64_t* checksum) {
  std::vector<int64_t> part((size_t)n_db, 0);
  std::vector<std::thread> th;
  const auto t0 = std::chrono::steady_clock::now();
  for (int i = 0; i < n_db; ++i) {
    th.emplace_back([&, i]() {
      const Database& db = *static_cast<Database*>(dbs[i]);
      if (which == 3) {
        Q3Args a;
        a.SEGMENT = kSegment[segment];
        a.DATE = date;
        for (const auto& r : run_q3(db, a)) part[(size_t)i] += r.revenue_raw;
      } else {
        Q1Args a;
        a.DELTA = std::to_string(delta_days);
        for (const auto& r : run_q1(db, a)) part[(size_t)i] += r.count_order;
      }
    });
  }
  for (auto& t : th) t.join();
  const double ms = ms_since(t0);
  int64_t s = 0;
  for (auto v : part) s += v;
  if (checksum) *checksum = s;
  return ms;
}

// Captures what the reference prints on stdout (the PROFILE / COUNT lines of a
// -DTRACE build, bespoke_tpch/query_q3.cpp:116-141) between begin and end.
static std::ostringstream g_trace;
static std::streambuf* g_old_cout = nullptr;

void ref_trace_begin() {
  g_trace.str("");
  g_old_cout = std::cout.rdbuf(g_trace.rdbuf());
}

int ref_trace_end(char* buf, int len) {
  if (g_old_cout) std::cout.rdbuf(g_old_cout);
  g_old_cout = nullptr;
  const std::string s = g_trace.str();
  if (buf && len > 0) std::snprintf(buf, (size_t)len, "%s", s.c_str());
  return (int)s.size();
}

int ref_has_trace() {
#ifdef TRACE
  return 1;
#else
  return 0;
#endif
}

}  // extern "C"
