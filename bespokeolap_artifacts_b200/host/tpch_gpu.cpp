// Drop-in GPU host for the reference's TPC-H engine: load / build / query.
// See tpch_gpu.hpp for the contract.
#include "tpch_gpu.hpp"

#include "host_threads.cuh"  // the engine's host thread pool (plain C++)

#include <arrow/api.h>
#include <arrow/io/file.h>
#include <parquet/arrow/reader.h>

#include <malloc.h>

#include <algorithm>
#include <array>
#include <charconv>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <functional>
#include <future>
#include <iomanip>
#include <iostream>
#include <mutex>
#include <numeric>
#include <sstream>
#include <stdexcept>
#include <thread>
#include <unordered_map>

namespace bo_tpch {

// Days since 1970-01-01 of a proleptic Gregorian date (H. Hinnant's
// days_from_civil algorithm) and its inverse.
int64_t days_from_civil(int64_t y, unsigned m, unsigned d) {
  y -= m <= 2;
  const int64_t era = (y >= 0 ? y : y - 399) / 400;
  const unsigned yoe = static_cast<unsigned>(y - era * 400);
  const unsigned doy = (153 * (m > 2 ? m - 3 : m + 9) + 2) / 5 + d - 1;
  const unsigned doe = yoe * 365 + yoe / 4 - yoe / 100 + doy;
  return era * 146097 + static_cast<int64_t>(doe) - 719468;
}

void civil_from_days(int64_t z, int& y, unsigned& m, unsigned& d) {
  z += 719468;
  const int64_t era = (z >= 0 ? z : z - 146096) / 146097;
  const unsigned doe = static_cast<unsigned>(z - era * 146097);
  const unsigned yoe = (doe - doe / 1460 + doe / 36524 - doe / 146096) / 365;
  const int64_t yy = static_cast<int64_t>(yoe) + era * 400;
  const unsigned doy = doe - (365 * yoe + yoe / 4 - yoe / 100);
  const unsigned mp = (5 * doy + 2) / 153;
  d = doy - (153 * mp + 2) / 5 + 1;
  m = mp < 10 ? mp + 3 : mp - 9;
  y = static_cast<int>(yy + (m <= 2));
}

namespace {

constexpr int32_t kPriceScale = 100;
constexpr int32_t kDiscountScale = 100;

void check(bo_ctx* ctx, int rc, const char* what) {
  if (rc != BO_OK) {
    throw std::runtime_error(std::string(what) + ": " + (ctx ? bo_last_error(ctx) : "no context") + " (status " +
                             std::to_string(rc) + ")");
  }
}

// ------------------------------------------------------------- arrow input --
std::shared_ptr<arrow::Table> read_parquet(const std::string& path) {
  auto file = arrow::io::ReadableFile::Open(path);
  if (!file.ok()) throw std::runtime_error("cannot open " + path + ": " + file.status().ToString());
  auto reader = parquet::arrow::OpenFile(*file, arrow::default_memory_pool());
  if (!reader.ok()) throw std::runtime_error("cannot read parquet " + path + ": " + reader.status().ToString());
  auto table = (*reader)->ReadTable();
  if (!table.ok()) throw std::runtime_error("cannot read table " + path + ": " + table.status().ToString());
  return *table;
}

std::shared_ptr<arrow::ChunkedArray> column(const ParquetTables::ArrowTable& t, const char* name) {
  auto c = t ? t->GetColumnByName(name) : nullptr;
  if (!c) throw std::runtime_error(std::string("Missing column: ") + name);
  return c;
}

template <class ArrayT, class T, class F>
void each(const std::shared_ptr<arrow::ChunkedArray>& c, std::vector<T>& out, F conv) {
  for (const auto& chunk : c->chunks()) {
    const auto a = std::static_pointer_cast<ArrayT>(chunk);
    for (int64_t i = 0; i < a->length(); ++i) out.push_back(a->IsNull(i) ? T{} : conv(a->Value(i)));
  }
}

// Integer keys (int32 / int64 columns), nulls as 0.
std::vector<int32_t> int_values(const std::shared_ptr<arrow::ChunkedArray>& c) {
  std::vector<int32_t> out;
  out.reserve(c->length());
  switch (c->type()->id()) {
    case arrow::Type::INT32:
      each<arrow::Int32Array>(c, out, [](int32_t v) { return v; });
      break;
    case arrow::Type::INT64:
      each<arrow::Int64Array>(c, out, [](int64_t v) { return static_cast<int32_t>(v); });
      break;
    default:
      throw std::runtime_error("Unsupported integer column type: " + c->type()->ToString());
  }
  return out;
}

// Decimal values scaled to integers: llround(value * scale); a decimal column
// goes through its text form and a double, as the reference's builder converts
// it (bespoke_tpch/builder_impl.cpp:287-338), so both round identically.
std::vector<int32_t> scaled_values(const std::shared_ptr<arrow::ChunkedArray>& c, int32_t scale) {
  std::vector<int32_t> out;
  out.reserve(c->length());
  const double s = static_cast<double>(scale);
  auto r = [s](double v) { return static_cast<int32_t>(std::llround(v * s)); };
  switch (c->type()->id()) {
    case arrow::Type::DOUBLE:
      each<arrow::DoubleArray>(c, out, [&](double v) { return r(v); });
      break;
    case arrow::Type::FLOAT:
      each<arrow::FloatArray>(c, out, [&](float v) { return r(static_cast<double>(v)); });
      break;
    case arrow::Type::INT32:
      each<arrow::Int32Array>(c, out, [&](int32_t v) { return r(static_cast<double>(v)); });
      break;
    case arrow::Type::INT64:
      each<arrow::Int64Array>(c, out, [&](int64_t v) { return r(static_cast<double>(v)); });
      break;
    case arrow::Type::DECIMAL128:
      for (const auto& chunk : c->chunks()) {
        const auto a = std::static_pointer_cast<arrow::Decimal128Array>(chunk);
        for (int64_t i = 0; i < a->length(); ++i) out.push_back(a->IsNull(i) ? 0 : r(std::stod(a->FormatValue(i))));
      }
      break;
    case arrow::Type::DECIMAL256:
      for (const auto& chunk : c->chunks()) {
        const auto a = std::static_pointer_cast<arrow::Decimal256Array>(chunk);
        for (int64_t i = 0; i < a->length(); ++i) out.push_back(a->IsNull(i) ? 0 : r(std::stod(a->FormatValue(i))));
      }
      break;
    default:
      throw std::runtime_error("Unsupported numeric column type: " + c->type()->ToString());
  }
  return out;
}

// Dates as int16 day offsets from base_days (DATE32 / DATE64; nulls as 0).
std::vector<int16_t> date_offsets(const std::shared_ptr<arrow::ChunkedArray>& c, int32_t base_days) {
  std::vector<int16_t> out;
  out.reserve(c->length());
  for (const auto& chunk : c->chunks()) {
    if (chunk->type_id() == arrow::Type::DATE32) {
      const auto a = std::static_pointer_cast<arrow::Date32Array>(chunk);
      for (int64_t i = 0; i < a->length(); ++i)
        out.push_back(a->IsNull(i) ? int16_t(0) : static_cast<int16_t>(a->Value(i) - base_days));
    } else if (chunk->type_id() == arrow::Type::DATE64) {
      const auto a = std::static_pointer_cast<arrow::Date64Array>(chunk);
      for (int64_t i = 0; i < a->length(); ++i)
        out.push_back(a->IsNull(i) ? int16_t(0)
                                   : static_cast<int16_t>(static_cast<int32_t>(a->Value(i) / 86400000) - base_days));
    } else {
      throw std::runtime_error("Unsupported date type: " + chunk->type()->ToString());
    }
  }
  return out;
}

// Calls fn(value) for each value of a string column (strings, large strings
// or dictionary-encoded strings; nulls as the empty string).
template <class F>
void for_each_string(const std::shared_ptr<arrow::ChunkedArray>& c, F fn) {
  for (const auto& chunk : c->chunks()) {
    switch (chunk->type_id()) {
      case arrow::Type::STRING: {
        const auto a = std::static_pointer_cast<arrow::StringArray>(chunk);
        for (int64_t i = 0; i < a->length(); ++i) fn(a->IsNull(i) ? std::string_view() : a->GetView(i));
        break;
      }
      case arrow::Type::LARGE_STRING: {
        const auto a = std::static_pointer_cast<arrow::LargeStringArray>(chunk);
        for (int64_t i = 0; i < a->length(); ++i) fn(a->IsNull(i) ? std::string_view() : a->GetView(i));
        break;
      }
      case arrow::Type::DICTIONARY: {
        const auto a = std::static_pointer_cast<arrow::DictionaryArray>(chunk);
        const auto values = std::static_pointer_cast<arrow::StringArray>(a->dictionary());
        for (int64_t i = 0; i < a->length(); ++i)
          fn(a->IsNull(i) ? std::string_view() : values->GetView(a->GetValueIndex(i)));
        break;
      }
      default:
        throw std::runtime_error("Unsupported string column type: " + chunk->type()->ToString());
    }
  }
}

struct ViewHash {
  using is_transparent = void;
  size_t operator()(std::string_view v) const { return std::hash<std::string_view>{}(v); }
};

// Dictionary codes in first-appearance order.  Lookups take the row's view
// (no per-row string), and a run of equal values reuses the last code.
std::vector<uint16_t> dictionary_codes(const std::shared_ptr<arrow::ChunkedArray>& c, Dictionary& dict) {
  std::vector<uint16_t> codes;
  codes.reserve(c->length());
  std::unordered_map<std::string, uint16_t, ViewHash, std::equal_to<>> ids;
  std::string last;
  int32_t last_id = -1;
  for_each_string(c, [&](std::string_view sv) {
    if (last_id >= 0 && sv == last) {
      codes.push_back(static_cast<uint16_t>(last_id));
      return;
    }
    auto it = ids.find(sv);
    uint16_t id;
    if (it != ids.end()) {
      id = it->second;
    } else {
      if (dict.values.size() > 0xffff) throw std::runtime_error("Dictionary column exceeds uint16_t capacity");
      id = static_cast<uint16_t>(dict.values.size());
      ids.emplace(std::string(sv), id);
      dict.values.emplace_back(sv);
    }
    last.assign(sv);
    last_id = id;
    codes.push_back(id);
  });
  return codes;
}

// Concatenated values with offsets (the reference's StringColumn layout).
StringColumn string_column(const std::shared_ptr<arrow::ChunkedArray>& c) {
  StringColumn out;
  out.offsets.reserve(c->length() + 1);
  out.offsets.push_back(0);
  for_each_string(c, [&](std::string_view v) {
    out.data.append(v);
    if (out.data.size() > 0xffffffffull) throw std::runtime_error("String column exceeds 4 GiB");
    out.offsets.push_back(static_cast<uint32_t>(out.data.size()));
  });
  return out;
}

template <class T>
DeviceColumn upload(bo_ctx* ctx, const std::vector<T>& v) {
  DeviceColumn c;
  c.rows = static_cast<int64_t>(v.size());
  check(ctx, bo_device_alloc(ctx, std::max<size_t>(sizeof(T) * v.size(), 256), &c.ptr), "device alloc");
  if (!v.empty()) check(ctx, bo_copy_h2d(ctx, c.ptr, v.data(), sizeof(T) * v.size()), "upload");
  return c;
}

template <class T>
std::vector<T> permute(const std::vector<T>& v, const std::vector<uint32_t>& order) {
  std::vector<T> out(v.size());
  for (size_t i = 0; i < order.size(); ++i) out[i] = v[order[i]];
  return out;
}

std::string escape_csv(const std::string& v) {
  std::string out = "\"";
  for (char ch : v) {
    if (ch == '"') out.push_back('\\');
    out.push_back(ch);
  }
  out.push_back('"');
  return out;
}

// "YYYY-MM-DD" plus add_months, the day clamped to the target month's length
// (the reference's parse_date_offset(_add_*) helpers, e.g.
// bespoke_tpch/query_q10.cpp:47-75), as a day offset from base_days.
int16_t date_offset_of(const std::string& text, int32_t base_days, int add_months = 0) {
  int y = std::stoi(text.substr(0, 4));
  int m = std::stoi(text.substr(5, 2));
  int d = std::stoi(text.substr(8, 2));
  if (add_months) {
    int index = m - 1 + add_months;
    y += index / 12;
    index %= 12;
    if (index < 0) {
      index += 12;
      y -= 1;
    }
    m = index + 1;
    static const int kDays[] = {31, 28, 31, 30, 31, 30, 31, 31, 30, 31, 30, 31};
    const bool leap = (y % 4 == 0 && y % 100 != 0) || y % 400 == 0;
    const int dim = (m == 2 && leap) ? 29 : kDays[m - 1];
    d = std::min(d, dim);
  }
  return static_cast<int16_t>(static_cast<int32_t>(days_from_civil(y, (unsigned)m, (unsigned)d)) - base_days);
}

int32_t scaled_arg(const std::string& text, int32_t scale) {
  return static_cast<int32_t>(std::llround(std::stod(text) * static_cast<double>(scale)));
}

template <class T>
const T* col(const DeviceColumn& c) {
  return static_cast<const T*>(c.ptr);
}

}  // namespace

// ----------------------------------------------------------------- queries --
std::vector<Q1ResultRow> run_q1(const Database& db, const std::string& delta) {
  const int32_t delta_days = static_cast<int32_t>(std::stoi(delta));
  const int32_t cutoff = static_cast<int32_t>(days_from_civil(1998, 12, 1)) - delta_days - db.base_date_days;
  const size_t rf = db.returnflag.values.size(), ls = db.linestatus.values.size();
  const size_t groups = rf * ls;
  std::vector<Q1ResultRow> rows;
  if (groups == 0) return rows;
  if (groups > BO_Q1_MAX_GROUPS)
    throw std::runtime_error("Q1: " + std::to_string(groups) + " returnflag x linestatus groups, the GPU path holds " +
                             std::to_string(BO_Q1_MAX_GROUPS));
  bo_lineitem_cols c{col<int16_t>(db.l_shipdate), col<uint8_t>(db.l_returnflag_linestatus),
                     col<int32_t>(db.l_extendedprice), col<int32_t>(db.l_discounted_price),
                     col<uint8_t>(db.l_discount), col<uint8_t>(db.l_tax), col<int16_t>(db.l_quantity), db.n_lineitem};
  void* dev = db.scratch.ptr;
  check(db.ctx, bo_q1_lineitem_device(db.ctx, &c, static_cast<int16_t>(cutoff), static_cast<int32_t>(groups),
                                      static_cast<bo_q1_agg*>(dev)),
        "q1");
  std::vector<bo_q1_agg> agg(groups);
  check(db.ctx, bo_copy_d2h(db.ctx, agg.data(), dev, sizeof(bo_q1_agg) * groups), "q1 result");
  check(db.ctx, bo_check_errors(db.ctx), "q1");
  // Finalisation of bespoke_tpch/query_q1.cpp:233-274: integer totals to
  // doubles by the same expressions, non-empty groups, (returnflag, linestatus) order.
  for (size_t g = 0; g < groups; ++g) {
    const bo_q1_agg& a = agg[g];
    if (a.count == 0) continue;
    const __int128 charge = (static_cast<__int128>(a.sum_charge.hi) << 64) | a.sum_charge.lo;
    const double count = static_cast<double>(a.count);
    Q1ResultRow r;
    r.returnflag = db.returnflag.values[g / ls];
    r.linestatus = db.linestatus.values[g % ls];
    r.sum_qty = static_cast<double>(a.sum_qty) / kPriceScale;
    r.sum_base_price = static_cast<double>(a.sum_base_price) / kPriceScale;
    r.sum_disc_price = static_cast<double>(a.sum_disc_price) / kPriceScale;
    r.sum_charge = static_cast<double>(charge) / (static_cast<double>(kPriceScale) * kDiscountScale);
    r.avg_qty = r.sum_qty / count;
    r.avg_price = r.sum_base_price / count;
    r.avg_disc = static_cast<double>(a.sum_disc) / kDiscountScale / count;
    r.count_order = a.count;
    rows.push_back(std::move(r));
  }
  std::sort(rows.begin(), rows.end(), [](const Q1ResultRow& x, const Q1ResultRow& y) {
    return x.returnflag == y.returnflag ? x.linestatus < y.linestatus : x.returnflag < y.returnflag;
  });
  return rows;
}

std::vector<Q6ResultRow> run_q6(const Database& db, const std::string& date, const std::string& discount,
                                const std::string& quantity) {
  const int16_t start = date_offset_of(date, db.base_date_days);
  const int16_t end = date_offset_of(date, db.base_date_days, 12);
  const int32_t d = scaled_arg(discount, kDiscountScale);
  const int32_t q = scaled_arg(quantity, kPriceScale);
  bo_lineitem_cols c{};
  c.shipdate = col<int16_t>(db.l_shipdate);
  c.extendedprice = col<int32_t>(db.l_extendedprice);
  c.discount = col<uint8_t>(db.l_discount);
  c.quantity = col<int16_t>(db.l_quantity);
  c.n_rows = db.n_lineitem;
  void* dev = db.scratch.ptr;
  check(db.ctx, bo_q6_lineitem_device(db.ctx, &c, start, end, d - 1, d + 1, q, static_cast<bo_q6_result*>(dev)),
        "q6");
  bo_q6_result r{};
  check(db.ctx, bo_copy_d2h(db.ctx, &r, dev, sizeof(r)), "q6 result");
  check(db.ctx, bo_check_errors(db.ctx), "q6");
  return {Q6ResultRow{r.revenue_raw}};
}

namespace {
// fn(begin, end) over [0, n), split across host threads when n is large: the
// result rows gather host-resident strings of random customers, a loop bound
// by memory latency that more threads overlap.  The threads are created once
// per process (a pool that spins briefly between loops, then sleeps).
template <class F>
void for_row_ranges(int64_t n, const F& fn) {
  constexpr int64_t kRowsPerThread = 8192;
  static bo::HostPool pool(static_cast<int>(
      std::min<int64_t>(8, std::max<int64_t>(1, static_cast<int64_t>(std::thread::hardware_concurrency())))));
  const int64_t parts = std::min<int64_t>(pool.threads(), (n + kRowsPerThread - 1) / kRowsPerThread);
  if (parts <= 1) {
    fn(int64_t{0}, n);
    return;
  }
  pool.parallel_for(n, [&fn](int64_t lo, int64_t hi) { fn(lo, hi); }, 2 * kRowsPerThread);
}

// BO_QUERY_TRACE set: a query's phases (the GPU call with its result copy,
// the host-side row materialisation) on stderr, in microseconds.
class QueryTrace {
 public:
  explicit QueryTrace(const char* query) : query_(query), on_(std::getenv("BO_QUERY_TRACE") != nullptr) {}
  void mark(const char* phase) {
    if (!on_) return;
    const auto now = std::chrono::steady_clock::now();
    std::cerr << query_ << " " << phase << " us: "
              << std::chrono::duration_cast<std::chrono::microseconds>(now - last_).count() << "\n";
    last_ = now;
  }

 private:
  const char* query_;
  bool on_;
  std::chrono::steady_clock::time_point last_ = std::chrono::steady_clock::now();
};

// Room for `count` result records of type T in the Database's pinned buffer.
template <class T>
T* result_rows(const Database& db, int64_t count) {
  const size_t bytes = sizeof(T) * static_cast<size_t>(std::max<int64_t>(count, 1));
  if (bytes > db.result_host_bytes) {
    if (db.result_host) check(db.ctx, bo_host_free_pinned(db.ctx, db.result_host), "result buffer free");
    db.result_host = nullptr;
    db.result_host_bytes = 0;
    check(db.ctx, bo_host_alloc_pinned(db.ctx, bytes, &db.result_host), "result buffer alloc");
    db.result_host_bytes = bytes;
  }
  return static_cast<T*>(db.result_host);
}
}  // namespace

RowView<Q3ResultRow> run_q3(const Database& db, const std::string& segment, const std::string& date) {
  const int16_t d = date_offset_of(date, db.base_date_days);
  int32_t code = -1;
  for (size_t i = 0; i < db.mktsegment.values.size(); ++i)
    if (db.mktsegment.values[i] == segment) {
      code = static_cast<int32_t>(i);
      break;
    }
  bo_tpch_q3_tables t{};
  t.c_custkey = col<int32_t>(db.c_custkey);
  t.c_mktsegment = col<uint16_t>(db.c_mktsegment);
  t.n_customer = db.n_customer;
  t.custkey_bound = db.custkey_bound;
  t.o_orderkey = col<int32_t>(db.o_orderkey);
  t.o_custkey = col<int32_t>(db.o_custkey);
  t.o_orderdate = col<int16_t>(db.o_orderdate);
  t.o_shippriority = col<int32_t>(db.o_shippriority);
  t.n_orders = db.n_orders;
  t.orderkey_to_row = col<int32_t>(db.orderkey_to_row);
  t.n_orderkey_map = db.n_orderkey_map;
  t.l_orderkey = col<int32_t>(db.l_orderkey);
  t.l_shipdate = col<int16_t>(db.l_shipdate);
  t.l_discounted_price = col<int32_t>(db.l_discounted_price);
  t.n_lineitem = db.n_lineitem;
  QueryTrace trace("q3");
  bo_tpch_q3_row* out = result_rows<bo_tpch_q3_row>(db, db.n_orders);
  int64_t n = 0;
  check(db.ctx, bo_tpch_q3(db.ctx, &t, d, code, out, db.n_orders, &n), "q3");
  trace.mark("gpu");
  return RowView<Q3ResultRow>(out, static_cast<size_t>(n));
}

Q10Rows run_q10(const Database& db, const std::string& date) {
  const int16_t start = date_offset_of(date, db.base_date_days);
  const int16_t end = date_offset_of(date, db.base_date_days, 3);
  int32_t rf = -1;
  for (size_t i = 0; i < db.returnflag.values.size(); ++i)
    if (db.returnflag.values[i] == "R") {
      rf = static_cast<int32_t>(i);
      break;
    }
  if (rf < 0) return {};
  const int32_t ls_count = static_cast<int32_t>(db.linestatus.values.size());
  bo_tpch_q10_tables t{};
  t.o_orderkey = col<int32_t>(db.o_orderkey);
  t.o_custkey = col<int32_t>(db.o_custkey);
  t.o_orderdate = col<int16_t>(db.o_orderdate);
  t.o_li_begin = col<uint32_t>(db.o_li_begin);
  t.o_li_end = col<uint32_t>(db.o_li_end);
  t.n_orders = db.n_orders;
  t.l_orderkey = col<int32_t>(db.l_orderkey);
  t.l_returnflag_linestatus = col<uint8_t>(db.l_returnflag_linestatus);
  t.l_discounted_price = col<int32_t>(db.l_discounted_price);
  t.n_lineitem = db.n_lineitem;
  t.lineitem_orderkey_sorted = db.lineitem_orderkey_sorted ? 1 : 0;
  t.nation_bound = db.nation_bound;
  t.custkey_to_row = col<int32_t>(db.custkey_to_row);
  t.n_custkey_map = db.n_custkey_map;
  t.c_nationkey = col<int32_t>(db.c_nationkey);
  t.n_customer = db.n_customer;
  t.c_name_offsets = col<uint32_t>(db.c_name_offsets);
  t.c_address_offsets = col<uint32_t>(db.c_address_offsets);
  t.c_phone_offsets = col<uint32_t>(db.c_phone_offsets);
  t.c_comment_offsets = col<uint32_t>(db.c_comment_offsets);
  t.c_acctbal = col<int32_t>(db.c_acctbal_device);
  QueryTrace trace("q10");
  // The rows are finished on the device: its last kernel writes them, strings
  // resolved to these host columns, straight into the mapped result buffer.
  const bo_tpch_q10_host_strings hs{db.c_name.data.data(),    db.c_address.data.data(),
                                    db.c_phone.data.data(),   db.c_comment.data.data(),
                                    db.nation_name_str.data(), static_cast<int32_t>(db.nation_name_str.size()),
                                    0};
  Q10ResultRow* out = result_rows<Q10ResultRow>(db, db.n_custkey_map);
  int64_t n = 0;
  check(db.ctx,
        bo_tpch_q10_host_rows(db.ctx, &t, start, end, rf * ls_count, ls_count, &hs, out, db.n_custkey_map, &n),
        "q10");
  trace.mark("gpu");
  return Q10Rows(out, static_cast<size_t>(n));
}

std::vector<Q4ResultRow> run_q4(const Database& db, const std::string& date) {
  // query_q4.cpp:179-181: the window [DATE, DATE + 3 months).
  const int16_t start = date_offset_of(date, db.base_date_days);
  const int16_t end = date_offset_of(date, db.base_date_days, 3);
  bo_tpch_q4_tables t{};
  t.o_orderkey = col<int32_t>(db.o_orderkey);
  t.o_orderdate = col<int16_t>(db.o_orderdate);
  t.o_orderpriority = col<uint16_t>(db.o_orderpriority);
  t.o_li_begin = col<uint32_t>(db.o_li_begin);
  t.o_li_end = col<uint32_t>(db.o_li_end);
  t.n_orders = db.n_orders;
  t.l_orderkey = col<int32_t>(db.l_orderkey);
  t.l_commit_receipt = col<uint32_t>(db.l_commit_receipt);
  t.n_lineitem = db.n_lineitem;
  t.lineitem_orderkey_sorted = db.lineitem_orderkey_sorted ? 1 : 0;
  t.n_priorities = static_cast<int32_t>(db.orderpriority.values.size());
  std::vector<int64_t> counts(db.orderpriority.values.size(), 0);
  check(db.ctx, bo_tpch_q4(db.ctx, &t, start, end, counts.data()), "q4");
  // Non-empty priorities in code order, then by name (:321-346).
  std::vector<Q4ResultRow> rows;
  for (size_t c = 0; c < counts.size(); ++c)
    if (counts[c] != 0) rows.push_back(Q4ResultRow{db.orderpriority.values[c], counts[c]});
  std::sort(rows.begin(), rows.end(),
            [](const Q4ResultRow& a, const Q4ResultRow& b) { return a.orderpriority < b.orderpriority; });
  return rows;
}

std::vector<Q5ResultRow> run_q5(const Database& db, const std::string& region, const std::string& date) {
  // query_q5.cpp:204-240: the region's key, the window [DATE, DATE + 1 year),
  // the nations of the region by key (any nation row of the key in it).
  const auto it = db.region_key_by_name.find(region);
  if (it == db.region_key_by_name.end()) return {};
  const int32_t region_key = it->second;
  const int16_t start = date_offset_of(date, db.base_date_days);
  const int16_t end = date_offset_of(date, db.base_date_days, 12);
  const int32_t n_nations = db.nation_bound;
  std::vector<uint8_t> in_region(static_cast<size_t>(n_nations), 0);
  for (size_t i = 0; i < db.nation_key.size(); ++i)
    if (db.nation_key[i] >= 0 && db.nation_regionkey[i] == region_key) in_region[static_cast<size_t>(db.nation_key[i])] = 1;
  bo_tpch_q5_tables t{};
  t.o_orderkey = col<int32_t>(db.o_orderkey);
  t.o_orderdate = col<int16_t>(db.o_orderdate);
  t.o_cust_nation = col<int16_t>(db.o_cust_nation);
  t.o_li_begin = col<uint32_t>(db.o_li_begin);
  t.o_li_end = col<uint32_t>(db.o_li_end);
  t.n_orders = db.n_orders;
  t.l_orderkey = col<int32_t>(db.l_orderkey);
  t.l_supp_nation = col<int16_t>(db.l_supp_nation);
  t.l_discounted_price = col<int32_t>(db.l_discounted_price);
  t.n_lineitem = db.n_lineitem;
  t.lineitem_orderkey_sorted = db.lineitem_orderkey_sorted ? 1 : 0;
  t.n_nations = n_nations;
  std::vector<int64_t> revenue(static_cast<size_t>(n_nations), 0);
  check(db.ctx, bo_tpch_q5(db.ctx, &t, in_region.data(), start, end, revenue.data()), "q5");
  // Region nations with non-zero revenue, by revenue desc then name (:497-548).
  std::vector<Q5ResultRow> rows;
  for (size_t n = 0; n < revenue.size(); ++n)
    if (in_region[n] && revenue[n] != 0) rows.push_back(Q5ResultRow{db.nation_name[n], revenue[n]});
  std::sort(rows.begin(), rows.end(), [](const Q5ResultRow& a, const Q5ResultRow& b) {
    return a.revenue_raw != b.revenue_raw ? a.revenue_raw > b.revenue_raw : a.n_name < b.n_name;
  });
  return rows;
}

std::vector<Q7ResultRow> run_q7(const Database& db, const std::string& nation1, const std::string& nation2) {
  // query_q7.cpp:141-199: both names' keys (the first nation row of a name),
  // the window 1995-01-01 .. 1996-12-31, supplier tags by supplier row.
  auto key_of = [&](const std::string& name, int32_t& key) {
    for (size_t i = 0; i < db.nation_row_name.size(); ++i)
      if (db.nation_row_name[i] == name) {
        key = db.nation_key[i];
        return true;
      }
    return false;
  };
  int32_t n1 = 0, n2 = 0;
  if (!key_of(nation1, n1) || !key_of(nation2, n2)) return {};
  const bool same = n1 == n2;
  const int16_t start = date_offset_of("1995-01-01", db.base_date_days);
  const int16_t last = date_offset_of("1996-12-31", db.base_date_days);
  const int16_t year2 = date_offset_of("1996-01-01", db.base_date_days);
  int32_t max_suppkey = -1;
  for (int32_t k : db.s_suppkey) max_suppkey = std::max(max_suppkey, k);
  std::vector<int8_t> tag(max_suppkey >= 0 ? static_cast<size_t>(max_suppkey) + 1 : 0, int8_t(-1));
  for (size_t i = 0; i < db.s_suppkey.size(); ++i) {
    const int32_t k = db.s_suppkey[i];
    if (k < 0) continue;
    if (db.s_nationkey[i] == n1)
      tag[static_cast<size_t>(k)] = 0;
    else if (!same && db.s_nationkey[i] == n2)
      tag[static_cast<size_t>(k)] = 1;
  }
  bo_tpch_q7_tables t{};
  t.l_shipdate = col<int16_t>(db.l_shipdate);
  t.l_suppkey = col<int32_t>(db.l_suppkey);
  t.l_orderkey = col<int32_t>(db.l_orderkey);
  t.l_discounted_price = col<int32_t>(db.l_discounted_price);
  t.n_lineitem = db.n_lineitem;
  t.orderkey_to_row = col<int32_t>(db.orderkey_to_row);
  t.n_orderkey_map = db.n_orderkey_map;
  t.o_cust_nation = col<int16_t>(db.o_cust_nation);
  t.n_orders = db.n_orders;
  int64_t revenue[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  check(db.ctx,
        bo_tpch_q7(db.ctx, &t, tag.data(), static_cast<int64_t>(tag.size()), n1, n2, start, last, year2, revenue),
        "q7");
  // Rows per (supplier nation, customer nation, year) with a non-zero sum,
  // named by the first nation row of each key (:372-412).
  auto name_of = [&](int32_t key, const std::string** out) {
    for (size_t i = 0; i < db.nation_key.size(); ++i)
      if (db.nation_key[i] == key) {
        *out = &db.nation_row_name[i];
        return true;
      }
    return false;
  };
  const int32_t nations[2] = {n1, n2};
  const int count = same ? 1 : 2;
  std::vector<Q7ResultRow> rows;
  for (int s = 0; s < count; ++s)
    for (int c = 0; c < count; ++c) {
      if (same ? (s != 0 || c != 0) : s == c) continue;
      const std::string *sn = nullptr, *cn = nullptr;
      if (!name_of(nations[s], &sn) || !name_of(nations[c], &cn)) continue;
      for (int y = 0; y < 2; ++y) {
        const int64_t v = revenue[s * 4 + c * 2 + y];
        if (v != 0) rows.push_back(Q7ResultRow{*sn, *cn, y == 0 ? 1995 : 1996, v});
      }
    }
  std::sort(rows.begin(), rows.end(), [](const Q7ResultRow& a, const Q7ResultRow& b) {
    if (a.supp_nation != b.supp_nation) return a.supp_nation < b.supp_nation;
    if (a.cust_nation != b.cust_nation) return a.cust_nation < b.cust_nation;
    return a.l_year < b.l_year;
  });
  return rows;
}

std::vector<Q8ResultRow> run_q8(const Database& db, const std::string& nation, const std::string& region,
                                const std::string& type) {
  // query_q8.cpp:123-198: the region's and the nation's keys (first row of a
  // name), the window 1995-01-01 .. 1996-12-31, the region's nations, the
  // target nation's suppliers, the type's code.
  const auto rit = db.region_key_by_name.find(region);
  if (rit == db.region_key_by_name.end()) return {};
  int32_t target = 0;
  bool found = false;
  for (size_t i = 0; i < db.nation_row_name.size() && !found; ++i)
    if (db.nation_row_name[i] == nation) {
      target = db.nation_key[i];
      found = true;
    }
  if (!found) return {};
  const int16_t start = date_offset_of("1995-01-01", db.base_date_days);
  const int16_t last = date_offset_of("1996-12-31", db.base_date_days);
  const int16_t year2 = date_offset_of("1996-01-01", db.base_date_days);
  std::vector<uint8_t> in_region(static_cast<size_t>(db.nation_bound), 0);
  for (size_t i = 0; i < db.nation_key.size(); ++i)
    if (db.nation_key[i] >= 0 && db.nation_key[i] < db.nation_bound && db.nation_regionkey[i] == rit->second)
      in_region[static_cast<size_t>(db.nation_key[i])] = 1;
  int32_t max_suppkey = -1;
  for (int32_t k : db.s_suppkey) max_suppkey = std::max(max_suppkey, k);
  std::vector<uint8_t> supp(max_suppkey >= 0 ? static_cast<size_t>(max_suppkey) + 1 : 0, 0);
  for (size_t i = 0; i < db.s_suppkey.size(); ++i)
    if (db.s_suppkey[i] >= 0 && db.s_nationkey[i] == target) supp[static_cast<size_t>(db.s_suppkey[i])] = 1;
  int32_t type_code = -1;
  for (size_t c = 0; c < db.part_type.values.size(); ++c)
    if (db.part_type.values[c] == type) {
      type_code = static_cast<int32_t>(c);
      break;
    }
  bo_tpch_q8_tables t{};
  t.l_partkey = col<int32_t>(db.l_partkey);
  t.l_suppkey = col<int32_t>(db.l_suppkey);
  t.l_orderkey = col<int32_t>(db.l_orderkey);
  t.l_extendedprice = col<int32_t>(db.l_extendedprice);
  t.l_discount = col<uint8_t>(db.l_discount);
  t.n_lineitem = db.n_lineitem;
  t.orderkey_to_row = col<int32_t>(db.orderkey_to_row);
  t.n_orderkey_map = db.n_orderkey_map;
  t.o_custkey = col<int32_t>(db.o_custkey);
  t.o_orderdate = col<int16_t>(db.o_orderdate);
  t.n_orders = db.n_orders;
  t.c_custkey = col<int32_t>(db.c_custkey);
  t.c_nationkey = col<int32_t>(db.c_nationkey);
  t.n_customer = db.n_customer;
  t.max_custkey = db.custkey_bound - 1;
  t.max_partkey = db.max_partkey;
  t.p_partkey = col<int32_t>(db.p_partkey);
  t.p_type = col<uint16_t>(db.p_type);
  t.n_part = db.n_part;
  int64_t sums[4] = {0, 0, 0, 0};
  check(db.ctx,
        bo_tpch_q8(db.ctx, &t, in_region.data(), static_cast<int32_t>(in_region.size()), supp.data(),
                   static_cast<int64_t>(supp.size()), type_code, start, last, year2, sums),
        "q8");
  // One row per year with a non-zero total, share = nation / total (:364-378).
  std::vector<Q8ResultRow> rows;
  for (int y = 0; y < 2; ++y)
    if (sums[2 + y] != 0)
      rows.push_back(Q8ResultRow{1995 + y, static_cast<double>(sums[y]) / static_cast<double>(sums[2 + y])});
  return rows;
}

std::vector<Q22ResultRow> run_q22(const Database& db, const std::vector<std::string>& codes) {
  // query_q22.cpp:24-60 (add_code): NULL and one-character codes are
  // skipped; a code whose first two characters are digits is that numeric
  // prefix, any other its first two characters; repeats are dropped.
  uint8_t numeric[100] = {};
  std::vector<int32_t> numeric_codes;
  std::vector<std::string> extra;
  std::vector<uint16_t> extra_pairs;
  for (const auto& v : codes) {
    if (v == "<<NULL>>" || v.size() < 2) continue;
    if (v[0] >= '0' && v[0] <= '9' && v[1] >= '0' && v[1] <= '9') {
      const int32_t code = (v[0] - '0') * 10 + (v[1] - '0');
      if (!numeric[code]) {
        numeric[code] = 1;
        numeric_codes.push_back(code);
      }
      continue;
    }
    const uint16_t packed = static_cast<uint16_t>((static_cast<uint8_t>(v[0]) << 8) | static_cast<uint8_t>(v[1]));
    if (std::find(extra_pairs.begin(), extra_pairs.end(), packed) != extra_pairs.end()) continue;
    extra.push_back(v.substr(0, 2));
    extra_pairs.push_back(packed);
  }
  if (numeric_codes.empty() && extra.empty()) return {};
  bo_tpch_q22_tables t{};
  t.c_custkey = col<int32_t>(db.c_custkey);
  t.c_acctbal = col<int32_t>(db.c_acctbal_device);
  t.c_phone_prefix = col<uint8_t>(db.c_phone_prefix);
  t.c_phone_pair = col<uint32_t>(db.c_phone_pair);
  t.n_customer = db.n_customer;
  t.o_has_order = col<uint32_t>(db.o_has_order);
  t.n_order_custkeys = db.n_order_custkeys;
  int64_t counts[107] = {}, sums[107] = {};
  check(db.ctx,
        bo_tpch_q22(db.ctx, &t, numeric, extra_pairs.data(), static_cast<int32_t>(extra_pairs.size()), counts, sums),
        "q22");
  // Numeric classes in request order, then the extra prefixes; non-empty
  // ones, by country code (:490-530).
  std::vector<Q22ResultRow> rows;
  for (const int32_t c : numeric_codes)
    if (counts[c] != 0)
      rows.push_back(Q22ResultRow{std::string{static_cast<char>('0' + c / 10), static_cast<char>('0' + c % 10)},
                                  counts[c], sums[c]});
  for (size_t i = 0; i < extra.size(); ++i)
    if (counts[100 + i] != 0) rows.push_back(Q22ResultRow{extra[i], counts[100 + i], sums[100 + i]});
  std::sort(rows.begin(), rows.end(),
            [](const Q22ResultRow& a, const Q22ResultRow& b) { return a.cntrycode < b.cntrycode; });
  return rows;
}

std::vector<Q16ResultRow> run_q16(const Database& db, const std::string& brand, const std::string& type,
                                  const std::string sizes[8]) {
  // query_q16.cpp:185-221: sizes that are all digits ("" is 0, "<<NULL>>"
  // and other text are skipped); none: no rows.  Sizes above 50 set no bit.
  uint64_t size_mask = 0;
  bool any = false;
  for (int i = 0; i < 8; ++i) {
    const std::string& v = sizes[i];
    if (v == "<<NULL>>") continue;
    uint32_t parsed = 0;
    bool digits = true;
    for (char ch : v) {
      if (ch < '0' || ch > '9') {
        digits = false;
        break;
      }
      parsed = parsed * 10u + static_cast<uint32_t>(ch - '0');
    }
    if (!digits) continue;
    any = true;
    if (static_cast<int32_t>(parsed) >= 0 && parsed <= 50) size_mask |= 1ull << parsed;
  }
  // :223-231, :346-355: no part rows or no supplier rows, no rows.
  if (!any || db.n_part == 0 || db.s_suppkey.empty()) return {};
  if (db.brand_rank.size() != db.brand.values.size() || db.type_rank.size() != db.part_type.values.size())
    throw std::runtime_error("Q16: dictionaries too large for ranks");
  // :233-270: types starting with TYPE are banned; the brand equal to BRAND.
  std::vector<uint8_t> type_banned(db.part_type.values.size(), 0);
  for (size_t i = 0; i < type_banned.size(); ++i)
    type_banned[i] = db.part_type.values[i].compare(0, type.size(), type) == 0 && db.part_type.values[i].size() >= type.size();
  int32_t banned_brand = -1;
  for (size_t i = 0; i < db.brand.values.size(); ++i)
    if (db.brand.values[i] == brand) {
      banned_brand = static_cast<int32_t>(i);
      break;
    }
  bo_tpch_q16_tables t{};
  t.p_partkey = col<int32_t>(db.p_partkey);
  t.p_brand = col<uint16_t>(db.p_brand);
  t.p_type = col<uint16_t>(db.p_type);
  t.p_size = col<int32_t>(db.p_size);
  t.n_part = db.n_part;
  t.ps_partkey = col<int32_t>(db.ps_partkey);
  t.ps_suppkey = col<int32_t>(db.ps_suppkey);
  t.n_partsupp = db.n_partsupp;
  t.s_banned = col<uint8_t>(db.s_banned);
  t.n_banned = db.n_s_banned;
  bo_tpch_q16_params prm{};
  prm.size_mask = size_mask;
  prm.banned_brand = banned_brand;
  // :383-388: a partsupp row count that is a multiple of the part rows is walked by position.
  prm.rows_per_part = db.n_partsupp % db.n_part == 0 ? static_cast<int32_t>(db.n_partsupp / db.n_part) : 0;
  prm.n_brand = static_cast<int32_t>(db.brand.values.size());
  prm.n_type = static_cast<int32_t>(db.part_type.values.size());
  prm.brand_rank = db.brand_rank.data();
  prm.type_rank = db.type_rank.data();
  prm.type_banned = type_banned.data();
  bo_tpch_q16_row* out = result_rows<bo_tpch_q16_row>(db, db.n_part);
  int64_t n = 0;
  check(db.ctx, bo_tpch_q16(db.ctx, &t, &prm, out, db.n_part, &n), "q16");
  std::vector<Q16ResultRow> rows(static_cast<size_t>(n));
  for (int64_t i = 0; i < n; ++i) {
    const auto& r = out[static_cast<size_t>(i)];
    rows[static_cast<size_t>(i)] = Q16ResultRow{db.brand.values[static_cast<size_t>(r.brand_code)],
                                                db.part_type.values[static_cast<size_t>(r.type_code)], r.size,
                                                r.supplier_cnt};
  }
  return rows;
}

std::vector<Q20ResultRow> run_q20(const Database& db, const std::string& color, const std::string& date,
                                  const std::string& nation) {
  // query_q20.cpp:344-361: a NULL parameter or an unknown nation, no rows
  // (the nation's first row by name).
  if (color == "<<NULL>>" || date == "<<NULL>>" || nation == "<<NULL>>") return {};
  int32_t key = 0;
  bool found = false;
  for (size_t i = 0; i < db.nation_row_name.size() && !found; ++i)
    if (db.nation_row_name[i] == nation) {
      key = db.nation_key[i];
      found = true;
    }
  if (!found) return {};
  const int16_t start = date_offset_of(date, db.base_date_days);
  const int16_t end = date_offset_of(date, db.base_date_days, 12);
  bo_tpch_q20_tables t{};
  t.p_partkey = col<int32_t>(db.p_partkey);
  t.p_name = col<char>(db.p_name);
  t.p_name_offsets = col<uint32_t>(db.p_name_offsets);
  t.n_part = db.n_part;
  t.max_partkey = db.max_partkey;
  t.max_suppkey = db.s_max_suppkey;
  t.l_shipdate = col<int16_t>(db.l_shipdate);
  t.l_partkey = col<int32_t>(db.l_partkey);
  t.l_suppkey = col<int32_t>(db.l_suppkey);
  t.l_supp_nation = col<int16_t>(db.l_supp_nation);
  t.l_quantity = col<int16_t>(db.l_quantity);
  t.n_lineitem = db.n_lineitem;
  t.ps_partkey = col<int32_t>(db.ps_partkey);
  t.ps_suppkey = col<int32_t>(db.ps_suppkey);
  t.ps_availqty = col<int32_t>(db.ps_availqty);
  t.n_partsupp = db.n_partsupp;
  t.ps_part_begin = col<int32_t>(db.ps_part_begin);
  t.n_ps_part_keys = db.n_ps_part_keys;
  t.s_nation_by_key = col<int16_t>(db.s_nation_by_key);
  t.s_suppkey = col<int32_t>(db.s_suppkey_device);
  t.s_nationkey = col<int32_t>(db.s_nationkey_device);
  t.s_row_by_name = col<int32_t>(db.s_row_by_name);
  t.n_supplier = static_cast<int64_t>(db.s_suppkey.size());
  int32_t* out = result_rows<int32_t>(db, t.n_supplier);
  int64_t n = 0;
  check(db.ctx,
        bo_tpch_q20(db.ctx, &t, color.data(), static_cast<int32_t>(color.size()), key, start, end, out, t.n_supplier,
                    &n),
        "q20");
  std::vector<Q20ResultRow> rows(static_cast<size_t>(n));
  for (int64_t i = 0; i < n; ++i) {
    const size_t r = static_cast<size_t>(out[static_cast<size_t>(i)]);
    rows[static_cast<size_t>(i)] = Q20ResultRow{db.s_name.view(r), db.s_address.view(r)};
  }
  return rows;
}

std::vector<Q2ResultRow> run_q2(const Database& db, const std::string& size, const std::string& type,
                                const std::string& region) {
  // query_q2.cpp:149-157: SIZE as std::stoi reads it; an unknown region, no rows.
  const int32_t target_size = std::stoi(size);
  const auto it = db.region_key_by_name.find(region);
  if (it == db.region_key_by_name.end()) return {};
  const int32_t region_key = it->second;
  // :166-183: nations by key below the row count; in the region when any row
  // of the key is.
  const size_t n_nation = db.nation_key.size();
  std::vector<uint8_t> nation_ok(n_nation, 0);
  for (size_t i = 0; i < n_nation; ++i)
    if (db.nation_key[i] >= 0 && static_cast<size_t>(db.nation_key[i]) < n_nation &&
        db.nation_regionkey[i] == region_key)
      nation_ok[static_cast<size_t>(db.nation_key[i])] = 1;
  // :214-230: types ending in TYPE.
  std::vector<uint8_t> type_ok(db.part_type.values.size(), 0);
  for (size_t i = 0; i < type_ok.size(); ++i) {
    const std::string& v = db.part_type.values[i];
    type_ok[i] = v.size() >= type.size() && v.compare(v.size() - type.size(), type.size(), type) == 0;
  }
  bo_tpch_q2_tables t{};
  t.p_size = col<int32_t>(db.p_size);
  t.p_type = col<uint16_t>(db.p_type);
  t.p_mfgr = col<uint16_t>(db.p_mfgr);
  t.n_part = db.n_part;
  t.ps_suppkey = col<int32_t>(db.ps_suppkey);
  t.ps_supplycost = col<int32_t>(db.ps_supplycost);
  t.n_partsupp = db.n_partsupp;
  t.ps_part_begin = col<int32_t>(db.ps_part_begin);
  t.n_ps_part_keys = db.n_ps_part_keys;
  t.s_nation_idx = col<int32_t>(db.s_nation_idx_device);
  t.s_rank = col<uint32_t>(db.s_rank);
  t.n_supplier = static_cast<int64_t>(db.s_suppkey.size());
  const int64_t cap = std::max<int64_t>(db.n_partsupp, 0);
  bo_tpch_q2_row* out = result_rows<bo_tpch_q2_row>(db, cap);
  int64_t n = 0;
  check(db.ctx,
        bo_tpch_q2(db.ctx, &t, target_size, type_ok.data(), static_cast<int32_t>(type_ok.size()), nation_ok.data(),
                   static_cast<int32_t>(n_nation), out, cap, &n),
        "q2");
  std::vector<Q2ResultRow> rows(static_cast<size_t>(n));
  for (int64_t i = 0; i < n; ++i) {
    const auto& o = out[static_cast<size_t>(i)];
    const size_t srow = static_cast<size_t>(o.supplier_row);
    const int32_t idx = db.s_nation_idx[srow];
    rows[static_cast<size_t>(i)] =
        Q2ResultRow{db.s_acctbal[srow],
                    db.s_name.view(srow),
                    idx >= 0 ? std::string_view(db.nation_name_by_idx[static_cast<size_t>(idx)]) : std::string_view(),
                    o.partkey,
                    db.mfgr.values[static_cast<size_t>(o.mfgr_code)],
                    db.s_address.view(srow),
                    db.s_phone.view(srow),
                    db.s_comment.view(srow)};
  }
  return rows;
}

std::vector<Q11ResultRow> run_q11(const Database& db, const std::string& nation, const std::string& fraction) {
  // query_q11.cpp:112-143: the nation's key (first nation row of the name),
  // FRACTION as a double, the nation's suppliers by key.
  int32_t key = 0;
  bool found = false;
  for (size_t i = 0; i < db.nation_row_name.size() && !found; ++i)
    if (db.nation_row_name[i] == nation) {
      key = db.nation_key[i];
      found = true;
    }
  if (!found) return {};
  const double frac = std::stod(fraction);
  int32_t max_suppkey = -1;
  for (int32_t k : db.s_suppkey) max_suppkey = std::max(max_suppkey, k);
  std::vector<uint8_t> in_nation(max_suppkey >= 0 ? static_cast<size_t>(max_suppkey) + 1 : 0, 0);
  for (size_t i = 0; i < db.s_suppkey.size(); ++i)
    if (db.s_nationkey[i] == key && db.s_suppkey[i] >= 0) in_nation[static_cast<size_t>(db.s_suppkey[i])] = 1;
  if (db.n_partsupp == 0) return {};
  bo_tpch_q11_tables t{};
  t.ps_partkey = col<int32_t>(db.ps_partkey);
  t.ps_suppkey = col<int32_t>(db.ps_suppkey);
  t.ps_value = col<int32_t>(db.ps_value);
  t.n_partsupp = db.n_partsupp;
  t.min_partkey = db.ps_min_partkey;
  t.max_partkey = db.ps_max_partkey;
  const int64_t range = static_cast<int64_t>(db.ps_max_partkey) - db.ps_min_partkey + 1;
  // :180-215 on the device: non-zero part sums above total * FRACTION, by
  // value desc then partkey.
  bo_tpch_q11_row* out = result_rows<bo_tpch_q11_row>(db, range);
  int64_t n = 0;
  check(db.ctx,
        bo_tpch_q11_rows(db.ctx, &t, in_nation.data(), static_cast<int64_t>(in_nation.size()), frac, out, range, &n),
        "q11");
  std::vector<Q11ResultRow> rows(static_cast<size_t>(n));
  for (int64_t i = 0; i < n; ++i) rows[static_cast<size_t>(i)] = Q11ResultRow{out[i].ps_partkey, out[i].value_raw};
  return rows;
}

std::vector<Q15ResultRow> run_q15(const Database& db, const std::string& date) {
  // query_q15.cpp:223-244: the quarter [DATE, DATE + 3 months), totals per
  // suppkey up to the largest supplier key.
  const int16_t start = date_offset_of(date, db.base_date_days);
  const int16_t end = date_offset_of(date, db.base_date_days, 3);
  int32_t max_suppkey = -1;
  for (int32_t k : db.s_suppkey) max_suppkey = std::max(max_suppkey, k);
  const int64_t n_supp = std::max<int64_t>(static_cast<int64_t>(max_suppkey) + 1, 1);
  bo_tpch_q15_tables t{};
  t.l_shipdate = col<int16_t>(db.l_shipdate);
  t.l_suppkey = col<int32_t>(db.l_suppkey);
  t.l_discounted_price = col<int32_t>(db.l_discounted_price);
  t.n_lineitem = db.n_lineitem;
  std::vector<int64_t> revenue(static_cast<size_t>(n_supp), 0);
  int64_t shipped = 0;
  check(db.ctx, bo_tpch_q15(db.ctx, &t, n_supp, start, end, revenue.data(), &shipped), "q15");
  // :454-530: nothing shipped, or no positive total: no rows; else the
  // suppliers (last row of a key) whose total is the largest, by suppkey.
  if (shipped == 0) return {};
  int64_t max_revenue = 0;
  for (int64_t v : revenue)
    if (v > 0) max_revenue = std::max(max_revenue, v);
  if (max_revenue == 0) return {};
  std::vector<int32_t> row_of(revenue.size(), -1);
  for (size_t i = 0; i < db.s_suppkey.size(); ++i)
    if (db.s_suppkey[i] >= 0 && static_cast<size_t>(db.s_suppkey[i]) < row_of.size())
      row_of[static_cast<size_t>(db.s_suppkey[i])] = static_cast<int32_t>(i);
  std::vector<Q15ResultRow> rows;
  for (size_t k = 0; k < revenue.size(); ++k) {
    if (revenue[k] != max_revenue || row_of[k] < 0) continue;
    const size_t r = static_cast<size_t>(row_of[k]);
    rows.push_back(Q15ResultRow{static_cast<int32_t>(k), db.s_name.view(r), db.s_address.view(r), db.s_phone.view(r),
                                revenue[k]});
  }
  return rows;
}

std::vector<Q9ResultRow> run_q9(const Database& db, const std::string& color) {
  // query_q9.cpp:188-226: the years of the orders' date span (no orders: no rows).
  if (db.n_orders == 0 || db.o_max_date < db.o_min_date) return {};
  const int32_t n_dates = static_cast<int32_t>(db.o_max_date) - db.o_min_date + 1;
  std::vector<int16_t> year_by_date(static_cast<size_t>(n_dates));
  for (int32_t i = 0; i < n_dates; ++i) {
    int y = 0;
    unsigned m = 0, d = 0;
    civil_from_days(static_cast<int64_t>(db.base_date_days) + db.o_min_date + i, y, m, d);
    year_by_date[static_cast<size_t>(i)] = static_cast<int16_t>(y);
  }
  const int32_t first_year = year_by_date.front(), last_year = year_by_date.back();
  const int32_t year_span = last_year - first_year + 1;
  check(db.ctx,
        bo_tpch_order_years(db.ctx, col<int32_t>(db.orderkey_to_row), db.n_orderkey_map, col<int16_t>(db.o_orderdate),
                            db.n_orders, db.o_min_date, year_by_date.data(), n_dates, first_year,
                            static_cast<uint8_t*>(db.o_year_by_key.ptr)),
        "q9 order years");
  // Groups (supplier nation, year) over nationkeys 0 .. the largest nation
  // row key (query_q9.cpp:153-163, 310-312).
  int32_t max_nationkey = 0;
  for (int32_t k : db.nation_key) max_nationkey = std::max(max_nationkey, k);
  std::vector<std::string> name_of(static_cast<size_t>(max_nationkey) + 1);
  for (size_t i = 0; i < db.nation_key.size(); ++i)
    if (db.nation_key[i] >= 0) name_of[static_cast<size_t>(db.nation_key[i])] = db.nation_row_name[i];
  const int32_t nation_bound = max_nationkey + 1;
  std::vector<int64_t> totals(static_cast<size_t>(nation_bound) * year_span);
  std::vector<uint8_t> used(totals.size());
  bo_tpch_q9_tables t{};
  t.l_partkey = col<int32_t>(db.l_partkey);
  t.l_suppkey = col<int32_t>(db.l_suppkey);
  t.l_orderkey = col<int32_t>(db.l_orderkey);
  t.l_quantity = col<int16_t>(db.l_quantity);
  t.l_discounted_price = col<int32_t>(db.l_discounted_price);
  t.l_supp_nation = col<int16_t>(db.l_supp_nation);
  t.n_lineitem = db.n_lineitem;
  t.p_name = col<char>(db.p_name);
  t.p_name_offsets = col<uint32_t>(db.p_name_offsets);
  t.p_partkey = col<int32_t>(db.p_partkey);
  t.n_part = db.n_part;
  t.ps_suppkey = col<int32_t>(db.ps_suppkey);
  t.ps_supplycost = col<int32_t>(db.ps_supplycost);
  t.ps_part_begin = col<int32_t>(db.ps_part_begin);
  t.n_part_keys = db.n_ps_part_keys;
  t.slots_per_part = db.ps_slots_per_part;
  t.o_year_by_key = static_cast<const uint8_t*>(db.o_year_by_key.ptr);
  t.n_orderkeys = db.n_orderkey_map;
  check(db.ctx,
        bo_tpch_q9(db.ctx, &t, color.data(), static_cast<int32_t>(color.size()), nation_bound, year_span,
                   totals.data(), used.data()),
        "q9");
  std::vector<Q9ResultRow> rows;
  for (int32_t n = 0; n < nation_bound; ++n) {
    if (name_of[static_cast<size_t>(n)].empty()) continue;
    for (int32_t y = 0; y < year_span; ++y) {
      const size_t g = static_cast<size_t>(n) * year_span + y;
      if (!used[g]) continue;
      rows.push_back(Q9ResultRow{name_of[static_cast<size_t>(n)], first_year + y, totals[g]});
    }
  }
  // ORDER BY nation, o_year DESC (query_q9.cpp:440-446)
  std::sort(rows.begin(), rows.end(), [](const Q9ResultRow& a, const Q9ResultRow& b) {
    if (a.nation != b.nation) return a.nation < b.nation;
    return a.o_year > b.o_year;
  });
  return rows;
}

std::vector<Q19ResultRow> run_q19(const Database& db, const std::string quantity[3], const std::string brand[3]) {
  // query_q19.cpp:133-157: every group off, or no partkey at all: one zero row.
  bool enabled[3], any = false;
  for (int g = 0; g < 3; ++g) any |= enabled[g] = quantity[g] != "<<NULL>>" && brand[g] != "<<NULL>>";
  const int32_t max_key = std::max(db.max_partkey, db.max_lineitem_partkey);
  if (!any || max_key < 0) return {Q19ResultRow{}};
  auto trim = [](std::string_view v) {
    while (!v.empty() && v.back() == ' ') v.remove_suffix(1);
    return v;
  };
  // Ship-mode codes: the last dictionary entry that trims to each mode; the
  // instruction code: the first that trims to it (query_q19.cpp:160-179).
  int32_t mode1 = -1, mode2 = -1, instruct = -1;
  for (size_t c = 0; c < db.shipmode.values.size(); ++c) {
    const auto v = trim(db.shipmode.values[c]);
    if (v == "AIR") mode1 = static_cast<int32_t>(c);
    else if (v == "AIR REG") mode2 = static_cast<int32_t>(c);
  }
  for (size_t c = 0; c < db.shipinstruct.values.size() && instruct < 0; ++c)
    if (trim(db.shipinstruct.values[c]) == "DELIVER IN PERSON") instruct = static_cast<int32_t>(c);
  int32_t brand_code[3], qty_low[3];
  const int32_t size_high[3] = {5, 10, 15};  // query_q19.cpp:221-240
  for (int g = 0; g < 3; ++g) {
    brand_code[g] = -1;
    qty_low[g] = 0;
    if (!enabled[g]) continue;
    qty_low[g] = static_cast<int32_t>(std::llround(std::stod(quantity[g]) * kPriceScale));
    for (size_t c = 0; c < db.brand.values.size(); ++c)
      if (db.brand.values[c] == brand[g]) brand_code[g] = static_cast<int32_t>(c);
  }
  // The three container lists (query_q19.cpp:203-208), as group bits per code.
  static const char* const kLists[3][4] = {{"SM CASE", "SM BOX", "SM PACK", "SM PKG"},
                                           {"MED BAG", "MED BOX", "MED PKG", "MED PACK"},
                                           {"LG CASE", "LG BOX", "LG PACK", "LG PKG"}};
  std::vector<uint8_t> groups(db.container.values.size(), 0);
  for (size_t c = 0; c < groups.size(); ++c)
    for (int g = 0; g < 3; ++g)
      for (const char* v : kLists[g])
        if (db.container.values[c] == v) groups[c] |= static_cast<uint8_t>(1u << g);
  bo_tpch_q19_tables t{};
  t.l_shipmode = col<uint16_t>(db.l_shipmode);
  t.l_shipinstruct = col<uint16_t>(db.l_shipinstruct);
  t.l_partkey = col<int32_t>(db.l_partkey);
  t.l_quantity = col<int16_t>(db.l_quantity);
  t.l_extendedprice = col<int32_t>(db.l_extendedprice);
  t.l_discount = col<uint8_t>(db.l_discount);
  t.n_lineitem = db.n_lineitem;
  t.p_row_by_key = col<int32_t>(db.p_row_by_key);
  t.n_part_keys = db.p_row_by_key.rows;
  t.p_brand = col<uint16_t>(db.p_brand);
  t.p_container = col<uint16_t>(db.p_container);
  t.p_size = col<int32_t>(db.p_size);
  t.n_part = db.n_part;
  t.n_mask = static_cast<int64_t>(max_key) + 1;
  int64_t revenue = 0;
  check(db.ctx,
        bo_tpch_q19(db.ctx, &t, brand_code, groups.data(), static_cast<int32_t>(groups.size()), size_high, qty_low,
                    mode1, mode2, instruct, &revenue),
        "q19");
  return {Q19ResultRow{revenue}};
}

std::vector<Q21ResultRow> run_q21(const Database& db, const std::string& nation) {
  // query_q21.cpp:148-190: a known nation (the first row of a name), an "F"
  // status code and a supplier key >= 0, else no rows.
  if (nation == "<<NULL>>") return {};
  int32_t target_nation = 0;
  bool found = false;
  for (size_t i = 0; i < db.nation_row_name.size() && !found; ++i)
    if (db.nation_row_name[i] == nation) {
      target_nation = db.nation_key[i];
      found = true;
    }
  if (!found) return {};
  int32_t final_code = -1;
  for (size_t c = 0; c < db.orderstatus.values.size() && final_code < 0; ++c)
    if (db.orderstatus.values[c] == "F") final_code = static_cast<int32_t>(c);
  if (final_code < 0) return {};
  int32_t max_suppkey = -1;
  for (int32_t k : db.s_suppkey) max_suppkey = std::max(max_suppkey, k);
  if (max_suppkey < 0) return {};
  // suppkey -> last supplier row; a target when any of its rows is of the nation
  std::vector<int32_t> row_of(static_cast<size_t>(max_suppkey) + 1, -1);
  std::vector<uint8_t> target(row_of.size(), 0);
  for (size_t r = 0; r < db.s_suppkey.size(); ++r) {
    const int32_t k = db.s_suppkey[r];
    if (k < 0) continue;
    row_of[static_cast<size_t>(k)] = static_cast<int32_t>(r);
    if (db.s_nationkey[r] == target_nation) target[static_cast<size_t>(k)] = 1;
  }
  bo_tpch_q21_tables t{};
  t.l_orderkey = col<int32_t>(db.l_orderkey);
  t.l_suppkey = col<int32_t>(db.l_suppkey);
  t.l_commit_receipt = col<uint32_t>(db.l_commit_receipt);
  t.n_lineitem = db.n_lineitem;
  t.o_orderkey = col<int32_t>(db.o_orderkey);
  t.o_orderstatus = col<uint16_t>(db.o_orderstatus);
  t.o_li_begin = col<uint32_t>(db.o_li_begin);
  t.o_li_end = col<uint32_t>(db.o_li_end);
  t.n_orders = db.n_orders;
  t.lineitem_orderkey_sorted = db.lineitem_orderkey_sorted ? 1 : 0;
  std::vector<int64_t> waits(row_of.size());
  check(db.ctx, bo_tpch_q21(db.ctx, &t, final_code, target.data(), max_suppkey, waits.data()), "q21");
  std::vector<Q21ResultRow> rows;
  for (size_t k = 0; k < waits.size(); ++k) {
    if (waits[k] == 0 || row_of[k] < 0) continue;
    rows.push_back(Q21ResultRow{db.s_name.view(static_cast<size_t>(row_of[k])), waits[k]});
  }
  // ORDER BY numwait DESC, s_name (query_q21.cpp:374-385)
  std::sort(rows.begin(), rows.end(), [](const Q21ResultRow& a, const Q21ResultRow& b) {
    if (a.numwait != b.numwait) return a.numwait > b.numwait;
    return a.s_name < b.s_name;
  });
  return rows;
}

std::vector<Q17ResultRow> run_q17(const Database& db, const std::string& brand, const std::string& container) {
  // query_q17.cpp:125-155: NULL arguments, no parts, or an unknown brand or
  // container give a zero row.
  if (brand == "<<NULL>>" || container == "<<NULL>>" || db.max_partkey < 0) return {Q17ResultRow{}};
  auto code_of = [](const Dictionary& d, const std::string& v) {
    for (size_t c = 0; c < d.values.size(); ++c)
      if (d.values[c] == v) return static_cast<int32_t>(c);
    return int32_t(-1);
  };
  const int32_t b = code_of(db.brand, brand), c = code_of(db.container, container);
  if (b < 0 || c < 0) return {Q17ResultRow{}};
  bo_tpch_q17_tables t{};
  t.l_partkey = col<int32_t>(db.l_partkey);
  t.l_quantity = col<int16_t>(db.l_quantity);
  t.l_extendedprice = col<int32_t>(db.l_extendedprice);
  t.n_lineitem = db.n_lineitem;
  t.p_partkey = col<int32_t>(db.p_partkey);
  t.p_brand = col<uint16_t>(db.p_brand);
  t.p_container = col<uint16_t>(db.p_container);
  t.n_part = db.n_part;
  t.max_partkey = db.max_partkey;
  int64_t sum = 0;
  check(db.ctx, bo_tpch_q17(db.ctx, &t, b, c, &sum), "q17");
  return {Q17ResultRow{sum}};
}

std::vector<Q14ResultRow> run_q14(const Database& db, const std::string& date) {
  // query_q14.cpp:189-200: the month [DATE, DATE + 1 month); no part keys: one zero row.
  const int16_t start = date_offset_of(date, db.base_date_days);
  const int16_t end = date_offset_of(date, db.base_date_days, 1);
  if (db.max_partkey < 0) return {Q14ResultRow{}};
  bo_tpch_q14_tables t{};
  t.l_shipdate = col<int16_t>(db.l_shipdate);
  t.l_partkey = col<int32_t>(db.l_partkey);
  t.l_discounted_price = col<int32_t>(db.l_discounted_price);
  t.n_lineitem = db.n_lineitem;
  t.p_promo_by_key = col<int8_t>(db.p_promo_by_key);
  t.n_promo_map = db.n_promo_map;
  int64_t sums[2] = {0, 0};
  check(db.ctx, bo_tpch_q14(db.ctx, &t, start, end, sums), "q14");
  Q14ResultRow row;  // :347-355
  if (sums[1] > 0) row.promo_revenue = 100.0 * static_cast<double>(sums[0]) / static_cast<double>(sums[1]);
  return {row};
}

std::vector<Q12ResultRow> run_q12(const Database& db, const std::string& shipmode1, const std::string& shipmode2,
                                  const std::string& date) {
  // query_q12.cpp:171-213: the window [DATE, DATE + 12 months), the two ship
  // modes' codes (the second only when it names another value) and the codes
  // of the two high priorities.
  const int16_t start = date_offset_of(date, db.base_date_days);
  const int16_t end = date_offset_of(date, db.base_date_days, 12);
  int32_t code1 = -1, code2 = -1;
  for (size_t c = 0; c < db.shipmode.values.size(); ++c) {
    if (db.shipmode.values[c] == shipmode1)
      code1 = static_cast<int32_t>(c);
    else if (db.shipmode.values[c] == shipmode2)
      code2 = static_cast<int32_t>(c);
  }
  if (code1 < 0 && code2 < 0) return {};
  int32_t high1 = -1, high2 = -1;
  for (size_t c = 0; c < db.orderpriority.values.size(); ++c) {
    if (db.orderpriority.values[c] == "1-URGENT")
      high1 = static_cast<int32_t>(c);
    else if (db.orderpriority.values[c] == "2-HIGH")
      high2 = static_cast<int32_t>(c);
  }
  bo_tpch_q12_tables t{};
  t.l_shipmode = col<uint16_t>(db.l_shipmode);
  t.l_commit_receipt = col<uint32_t>(db.l_commit_receipt);
  t.l_shipdate = col<int16_t>(db.l_shipdate);
  t.l_orderkey = col<int32_t>(db.l_orderkey);
  t.l_shard_max_shipdate = db.l_shard_max_shipdate.ptr ? col<int16_t>(db.l_shard_max_shipdate) : nullptr;
  t.n_lineitem = db.n_lineitem;
  t.orderkey_to_row = col<int32_t>(db.orderkey_to_row);
  t.n_orderkey_map = db.n_orderkey_map;
  t.o_orderpriority = col<uint16_t>(db.o_orderpriority);
  t.n_orders = db.n_orders;
  int64_t counts[4] = {0, 0, 0, 0};
  check(db.ctx, bo_tpch_q12(db.ctx, &t, code1, code2, high1, high2, start, end, counts), "q12");
  // Groups in code order, empty ones dropped, then by shipmode (:321-352).
  std::vector<Q12ResultRow> rows;
  for (size_t c = 0; c < db.shipmode.values.size(); ++c) {
    const int32_t code = static_cast<int32_t>(c);
    if (code != code1 && code != code2) continue;
    const int64_t high = code == code1 ? counts[0] : counts[2];
    const int64_t low = code == code1 ? counts[1] : counts[3];
    if (high == 0 && low == 0) continue;
    rows.push_back(Q12ResultRow{db.shipmode.values[c], high, low});
  }
  std::sort(rows.begin(), rows.end(),
            [](const Q12ResultRow& a, const Q12ResultRow& b) { return a.shipmode < b.shipmode; });
  return rows;
}

std::vector<Q13ResultRow> run_q13(const Database& db, const std::string& word1, const std::string& word2) {
  bo_tpch_q13_tables t{};
  t.o_comment = col<uint8_t>(db.o_comment);
  t.o_comment_offsets = col<uint32_t>(db.o_comment_offsets);
  t.o_custkey = col<int32_t>(db.o_custkey);
  t.n_orders = db.n_orders;
  t.c_custkey = col<int32_t>(db.c_custkey);
  t.n_customer = db.n_customer;
  t.n_count_map = std::max<int64_t>(db.custkey_bound, 1);
  const int64_t cap = db.n_orders + 1;  // distinct order counts
  bo_tpch_q13_row* out = result_rows<bo_tpch_q13_row>(db, cap);
  int64_t n = 0;
  check(db.ctx,
        bo_tpch_q13(db.ctx, &t, word1.data(), static_cast<int64_t>(word1.size()), word2.data(),
                    static_cast<int64_t>(word2.size()), out, cap, &n),
        "q13");
  std::vector<Q13ResultRow> rows(static_cast<size_t>(n));
  for (int64_t i = 0; i < n; ++i) rows[i] = Q13ResultRow{out[i].c_count, out[i].custdist};
  return rows;
}

std::vector<Q18ResultRow> run_q18(const Database& db, const std::string& quantity) {
  if (quantity == "<<NULL>>") return {};
  const int32_t threshold = scaled_arg(quantity, kPriceScale);
  int32_t max_key = db.max_lineitem_orderkey;
  if (db.n_orderkey_map > 0) max_key = std::max(max_key, static_cast<int32_t>(db.n_orderkey_map - 1));
  bo_tpch_q18_tables t{};
  t.o_orderkey = col<int32_t>(db.o_orderkey);
  t.o_custkey = col<int32_t>(db.o_custkey);
  t.o_orderdate = col<int16_t>(db.o_orderdate);
  t.o_totalprice = col<int32_t>(db.o_totalprice);
  t.n_orders = db.n_orders;
  t.l_orderkey = col<int32_t>(db.l_orderkey);
  t.l_quantity = col<int16_t>(db.l_quantity);
  t.n_lineitem = db.n_lineitem;
  t.custkey_to_row = col<int32_t>(db.custkey_to_row);
  t.n_custkey_map = db.n_custkey_map;
  t.n_customer = db.n_customer;
  t.orderkey_bound = max_key >= 0 ? static_cast<int64_t>(max_key) + 1 : 0;
  t.dense_orderkeys = db.dense_orderkeys ? 1 : 0;
  t.dense_custkeys = db.dense_custkeys ? 1 : 0;
  bo_tpch_q18_row* out = result_rows<bo_tpch_q18_row>(db, db.n_orders);
  int64_t n = 0;
  check(db.ctx, bo_tpch_q18(db.ctx, &t, threshold, out, db.n_orders, &n), "q18");
  std::vector<Q18ResultRow> rows(static_cast<size_t>(n));
  for_row_ranges(n, [&](int64_t lo, int64_t hi) {
    for (int64_t i = lo; i < hi; ++i) {
      const auto& g = out[i];
      auto& row = rows[i];
      row.c_name = db.c_name.view(static_cast<size_t>(g.cust_row));
      row.c_custkey = g.custkey;
      row.o_orderkey = g.orderkey;
      row.o_orderdate_offset = g.orderdate_offset;
      row.o_totalprice_raw = g.totalprice_raw;
      row.sum_qty_raw = g.sum_qty_raw;
    }
  });
  return rows;
}

// ------------------------------------------------------------------ output --
namespace {

std::string format_date(int32_t base_days, int16_t offset) {
  int y = 0;
  unsigned m = 0, d = 0;
  civil_from_days(base_days + offset, y, m, d);
  std::ostringstream date;
  date << std::setw(4) << std::setfill('0') << y << '-' << std::setw(2) << std::setfill('0') << m << '-'
       << std::setw(2) << std::setfill('0') << d;
  return date.str();
}

void append_csv_field(std::string& out, std::string_view v) {
  out.push_back('"');
  for (char ch : v) {
    if (ch == '"') out.push_back('\\');
    out.push_back(ch);
  }
  out.push_back('"');
}

// Sign, integer part and two decimals of a x100 value (query_q10.cpp:110-123).
void append_fixed_2(std::string& out, int64_t v) {
  if (v < 0) {
    out.push_back('-');
    v = -v;
  }
  char buf[32];
  const auto res = std::to_chars(std::begin(buf), std::end(buf), v / kPriceScale);
  out.append(buf, res.ptr);
  out.push_back('.');
  out.push_back(static_cast<char>('0' + (v % kPriceScale) / 10));
  out.push_back(static_cast<char>('0' + (v % kPriceScale) % 10));
}

}  // namespace

void write_q1_csv(const std::string& filename, const std::vector<Q1ResultRow>& rows) {
  std::ofstream out(filename);
  out << "l_returnflag,l_linestatus,sum_qty,sum_base_price,sum_disc_price,sum_charge,avg_qty,avg_price,avg_disc,"
         "count_order\n";
  out.setf(std::ios::fixed);
  out << std::setprecision(2);
  for (const auto& r : rows) {
    out << r.returnflag << ',' << r.linestatus << ',' << r.sum_qty << ',' << r.sum_base_price << ','
        << r.sum_disc_price << ',' << r.sum_charge << ',' << r.avg_qty << ',' << r.avg_price << ','
        << std::setprecision(4) << r.avg_disc << std::setprecision(2) << ',' << r.count_order << "\n";
  }
}

void write_q3_csv(const Database& db, const std::string& filename, const RowView<Q3ResultRow>& rows) {
  std::ofstream out(filename);
  out << "l_orderkey,revenue,o_orderdate,o_shippriority\n";
  out.setf(std::ios::fixed);
  out << std::setprecision(2);
  for (const auto& r : rows) {
    out << r.orderkey << ',' << static_cast<double>(r.revenue_raw) / kPriceScale << ','
        << format_date(db.base_date_days, r.orderdate_offset) << ',' << r.shippriority << "\n";
  }
}


void write_q10_csv(const std::string& filename, const Q10Rows& rows) {
  std::ofstream out(filename, std::ios::binary);
  std::string buf;
  buf.reserve(1 << 20);
  buf.append("c_custkey,c_name,revenue,c_acctbal,n_name,c_address,c_phone,c_comment\n");
  for (const auto& r : rows) {
    char ib[32];
    const auto res = std::to_chars(std::begin(ib), std::end(ib), r.custkey);
    buf.append(ib, res.ptr);
    buf.push_back(',');
    append_csv_field(buf, view_of(r.name));
    buf.push_back(',');
    append_fixed_2(buf, r.revenue_raw);
    buf.push_back(',');
    append_fixed_2(buf, r.acctbal_raw);
    buf.push_back(',');
    append_csv_field(buf, view_of(r.nation_name));
    buf.push_back(',');
    append_csv_field(buf, view_of(r.address));
    buf.push_back(',');
    append_csv_field(buf, view_of(r.phone));
    buf.push_back(',');
    append_csv_field(buf, view_of(r.comment));
    buf.push_back('\n');
    if (buf.size() >= (1u << 20)) {
      out.write(buf.data(), static_cast<std::streamsize>(buf.size()));
      buf.clear();
    }
  }
  out.write(buf.data(), static_cast<std::streamsize>(buf.size()));
}

void write_q4_csv(const std::string& filename, const std::vector<Q4ResultRow>& rows) {
  std::ofstream out(filename);  // query_q4.cpp:357-362
  out << "o_orderpriority,order_count\n";
  for (const auto& r : rows) out << escape_csv(r.orderpriority) << ',' << r.order_count << "\n";
}

void write_q5_csv(const std::string& filename, const std::vector<Q5ResultRow>& rows) {
  std::ofstream out(filename);  // query_q5.cpp:560-569
  out << "n_name,revenue\n";
  out.setf(std::ios::fixed);
  out << std::setprecision(2);
  for (const auto& r : rows)
    out << escape_csv(r.n_name) << ',' << static_cast<double>(r.revenue_raw) / static_cast<double>(kPriceScale) << "\n";
}

void write_q7_csv(const std::string& filename, const std::vector<Q7ResultRow>& rows) {
  std::ofstream out(filename);  // query_q7.cpp:425-435
  out << "supp_nation,cust_nation,l_year,revenue\n";
  out.setf(std::ios::fixed);
  out << std::setprecision(2);
  for (const auto& r : rows)
    out << escape_csv(r.supp_nation) << ',' << escape_csv(r.cust_nation) << ',' << r.l_year << ','
        << static_cast<double>(r.revenue_raw) / kPriceScale << "\n";
}

void write_q9_csv(const std::string& filename, const std::vector<Q9ResultRow>& rows) {
  std::ofstream out(filename);  // query_q9.cpp:449-460
  out << "nation,o_year,sum_profit\n";
  out.setf(std::ios::fixed);
  out << std::setprecision(2);
  for (const auto& r : rows)
    out << escape_csv(r.nation) << ',' << r.o_year << ',' << static_cast<double>(r.sum_profit_raw) / kPriceScale << "\n";
}

void write_q19_csv(const std::string& filename, const std::vector<Q19ResultRow>& rows) {
  std::ofstream out(filename);  // query_q19.cpp:340-351
  out << "revenue\n";
  out.setf(std::ios::fixed);
  out << std::setprecision(2);
  for (const auto& r : rows) out << static_cast<double>(r.revenue_raw) / (kPriceScale * kDiscountScale) << "\n";
}

void write_q21_csv(const std::string& filename, const std::vector<Q21ResultRow>& rows) {
  std::ofstream out(filename);  // query_q21.cpp:394-400
  out << "s_name,numwait\n";
  for (const auto& r : rows) out << escape_csv(std::string(r.s_name)) << ',' << r.numwait << "\n";
}

void write_q8_csv(const std::string& filename, const std::vector<Q8ResultRow>& rows) {
  std::ofstream out(filename);  // query_q8.cpp:382-389
  out << "o_year,mkt_share\n";
  out.setf(std::ios::fixed);
  out << std::setprecision(2);
  for (const auto& r : rows) out << r.o_year << "," << r.mkt_share << "\n";
}

void write_q22_csv(const std::string& filename, const std::vector<Q22ResultRow>& rows) {
  std::ofstream out(filename);  // query_q22.cpp:544-554
  out << "cntrycode,numcust,totacctbal\n";
  out.setf(std::ios::fixed);
  out << std::setprecision(2);
  for (const auto& r : rows)
    out << escape_csv(r.cntrycode) << ',' << r.numcust << ',' << static_cast<double>(r.totacctbal_raw) / kPriceScale
        << "\n";
}

void write_q16_csv(const std::string& filename, const std::vector<Q16ResultRow>& rows) {
  std::ofstream out(filename);  // query_q16.cpp:543-556
  out << "p_brand,p_type,p_size,supplier_cnt\n";
  for (const auto& r : rows)
    out << escape_csv(std::string(r.p_brand)) << ',' << escape_csv(std::string(r.p_type)) << ',' << r.p_size << ','
        << r.supplier_cnt << "\n";
}

void write_q20_csv(const std::string& filename, const std::vector<Q20ResultRow>& rows) {
  std::ofstream out(filename);  // query_q20.cpp:678-686
  out << "s_name,s_address\n";
  for (const auto& r : rows)
    out << escape_csv(std::string(r.s_name)) << ',' << escape_csv(std::string(r.s_address)) << "\n";
}

void write_q2_csv(const std::string& filename, const std::vector<Q2ResultRow>& rows) {
  std::ofstream out(filename);  // query_q2.cpp:432-454
  out << "s_acctbal,s_name,n_name,p_partkey,p_mfgr,s_address,s_phone,s_comment\n";
  out.setf(std::ios::fixed);
  out << std::setprecision(2);
  for (const auto& r : rows)
    out << static_cast<double>(r.s_acctbal_raw) / kPriceScale << ',' << escape_csv(std::string(r.s_name)) << ','
        << escape_csv(std::string(r.n_name)) << ',' << r.p_partkey << ',' << escape_csv(std::string(r.p_mfgr)) << ','
        << escape_csv(std::string(r.s_address)) << ',' << escape_csv(std::string(r.s_phone)) << ','
        << escape_csv(std::string(r.s_comment)) << "\n";
}

void write_q11_csv(const std::string& filename, const std::vector<Q11ResultRow>& rows) {
  std::ofstream out(filename);  // query_q11.cpp:226-234
  out << "ps_partkey,value\n";
  out.setf(std::ios::fixed);
  out << std::setprecision(2);
  for (const auto& r : rows) out << r.ps_partkey << ',' << static_cast<double>(r.value_raw) / kPriceScale << "\n";
}

void write_q15_csv(const std::string& filename, const std::vector<Q15ResultRow>& rows) {
  std::ofstream out(filename);  // query_q15.cpp:536-548
  out << "s_suppkey,s_name,s_address,s_phone,total_revenue\n";
  out.setf(std::ios::fixed);
  out << std::setprecision(2);
  for (const auto& r : rows)
    out << r.s_suppkey << ',' << escape_csv(std::string(r.s_name)) << ',' << escape_csv(std::string(r.s_address))
        << ',' << escape_csv(std::string(r.s_phone)) << ','
        << static_cast<double>(r.total_revenue_raw) / kPriceScale << "\n";
}

void write_q17_csv(const std::string& filename, const std::vector<Q17ResultRow>& rows) {
  std::ofstream out(filename);  // query_q17.cpp:311-321
  out << "avg_yearly\n";
  out.setf(std::ios::fixed);
  out << std::setprecision(2);
  for (const auto& r : rows)
    out << static_cast<double>(r.sum_extendedprice_raw) / (7.0 * static_cast<double>(kPriceScale)) << "\n";
}

void write_q14_csv(const std::string& filename, const std::vector<Q14ResultRow>& rows) {
  std::ofstream out(filename);  // query_q14.cpp:367-374
  out << "promo_revenue\n";
  out.setf(std::ios::fixed);
  out << std::setprecision(2);
  for (const auto& r : rows) out << r.promo_revenue << "\n";
}

void write_q12_csv(const std::string& filename, const std::vector<Q12ResultRow>& rows) {
  std::ofstream out(filename);  // query_q12.cpp:362-368
  out << "l_shipmode,high_line_count,low_line_count\n";
  for (const auto& r : rows) out << escape_csv(r.shipmode) << ',' << r.high_line_count << ',' << r.low_line_count << "\n";
}

void write_q13_csv(const std::string& filename, const std::vector<Q13ResultRow>& rows) {
  std::ofstream out(filename);
  out << "c_count,custdist\n";
  for (const auto& r : rows) out << r.c_count << ',' << r.custdist << "\n";
}

void write_q18_csv(const Database& db, const std::string& filename, const std::vector<Q18ResultRow>& rows) {
  std::ofstream out(filename);
  out << "c_name,c_custkey,o_orderkey,o_orderdate,o_totalprice,sum(l_quantity)\n";
  out.setf(std::ios::fixed);
  out << std::setprecision(2);
  for (const auto& r : rows) {
    out << escape_csv(std::string(r.c_name)) << ',' << r.c_custkey << ',' << r.o_orderkey << ','
        << format_date(db.base_date_days, r.o_orderdate_offset) << ','
        << static_cast<double>(r.o_totalprice_raw) / kPriceScale << ','
        << static_cast<double>(r.sum_qty_raw) / kPriceScale << "\n";
  }
}

void write_q6_csv(const std::string& filename, const std::vector<Q6ResultRow>& rows) {
  std::ofstream out(filename);
  out << "revenue\n";
  out.setf(std::ios::fixed);
  out << std::setprecision(2);
  for (const auto& r : rows)
    out << static_cast<double>(r.revenue_raw) / (static_cast<double>(kPriceScale) * kDiscountScale) << "\n";
}

}  // namespace bo_tpch

using namespace bo_tpch;

Database::~Database() {
  if (!ctx) return;
  DeviceColumn* cols[] = {&l_orderkey, &l_shipdate, &l_returnflag_linestatus, &l_extendedprice, &l_discounted_price,
                          &l_discount, &l_tax, &l_quantity, &o_orderkey, &o_custkey, &o_orderdate,
                          &o_shippriority, &o_totalprice, &orderkey_to_row, &o_li_begin, &o_li_end,
                          &o_comment, &o_comment_offsets, &o_orderpriority, &l_shipmode, &l_commit_receipt,
                          &l_shard_max_shipdate, &l_partkey, &p_promo_by_key, &l_supp_nation, &o_cust_nation,
                          &p_partkey, &p_brand, &p_container, &l_suppkey, &p_type, &c_acctbal_device,
                          &c_phone_prefix, &c_phone_pair, &o_has_order, &ps_partkey, &ps_suppkey, &ps_value,
                          &c_custkey, &c_mktsegment, &c_nationkey, &custkey_to_row, &scratch, &p_name,
                          &p_name_offsets, &ps_supplycost, &ps_part_begin, &o_year_by_key, &l_shipinstruct,
                          &p_size, &p_row_by_key, &o_orderstatus, &c_name_offsets, &c_address_offsets,
                          &c_phone_offsets, &c_comment_offsets, &s_comment_chars, &s_comment_offsets,
                          &s_suppkey_device, &s_banned, &s_nation_by_key, &s_nationkey_device,
                          &s_row_by_name, &ps_availqty, &s_nation_idx_device, &s_rank, &p_mfgr};
  for (auto* c : cols)
    if (c->ptr) bo_device_free(ctx, c->ptr);
  if (result_host) bo_host_free_pinned(ctx, result_host);
  bo_destroy(ctx);
}

// ---------------------------------------------------------- entry points --
namespace {
int device_from_env() {
  const char* e = std::getenv("BO_DEVICE");
  return e ? std::atoi(e) : 0;
}

// Device start-up begun by load() and awaited by build().
std::mutex g_device_init_mu;
std::future<int> g_device_init;

void start_device_init() {
  std::lock_guard<std::mutex> lock(g_device_init_mu);
  if (!g_device_init.valid())
    g_device_init = std::async(std::launch::async, [d = device_from_env()] { return bo_device_init(d); });
}

void await_device_init() {
  std::lock_guard<std::mutex> lock(g_device_init_mu);
  if (g_device_init.valid()) g_device_init.get();  // bo_create reports any failure itself
}
}  // namespace

ParquetTables* load(std::string path) {
  // The CUDA context is created on a background thread while the files are
  // read (the eight files themselves are read concurrently).
  start_device_init();
  auto* t = new ParquetTables{};
  auto read = [&path](const char* name) {
    return std::async(std::launch::async, [file = path + name] { return read_parquet(file); });
  };
  auto customer = read("customer.parquet");
  auto lineitem = read("lineitem.parquet");
  auto nation = read("nation.parquet");
  auto orders = read("orders.parquet");
  auto part = read("part.parquet");
  auto partsupp = read("partsupp.parquet");
  auto region = read("region.parquet");
  auto supplier = read("supplier.parquet");
  try {
    t->customer = customer.get();
    t->lineitem = lineitem.get();
    t->nation = nation.get();
    t->orders = orders.get();
    t->part = part.get();
    t->partsupp = partsupp.get();
    t->region = region.get();
    t->supplier = supplier.get();
  } catch (...) {
    delete t;
    throw;
  }
  return t;
}

namespace {

// Host-side storage-plan columns of one table, derived before the upload.
struct LineitemHost {
  std::vector<int32_t> orderkey, price, dprice, partkey, suppkey;
  std::vector<int16_t> ship, q16, shard_max_ship, supp_nation;
  std::vector<uint8_t> code, d8, t8;
  std::vector<uint16_t> shipmode, shipinstruct;
  std::vector<uint32_t> commit_receipt;
  Dictionary returnflag, linestatus, shipmode_dict, shipinstruct_dict;
  int32_t max_partkey = -1;
  bool orderkey_sorted = true;
  int32_t max_orderkey = -1;
};

struct OrdersHost {
  std::vector<int32_t> okey, ckey, prio, total, map;
  std::vector<uint16_t> priority, status;
  Dictionary priority_dict, status_dict;
  std::vector<int16_t> odate;
  std::vector<uint8_t> comment_bytes;
  std::vector<uint32_t> comment_offsets;
};

struct CustomerHost {
  std::vector<int32_t> ckey, nkey, map, acctbal;
  std::vector<uint16_t> seg;
  Dictionary mktsegment;
  int32_t max_key = 0;
  StringColumn name, address, phone, comment;
};

// lineitem: the storage-plan columns of bespoke_tpch/builder_impl.cpp:456-577.
// Each lineitem's supplier nation (bespoke_tpch/builder_impl.cpp:838-853):
// supplier's nationkey_by_suppkey (:719-742, last row of a key wins), -1 for
// suppkeys without a supplier.
std::vector<int16_t> supplier_nations(const ParquetTables::ArrowTable& L, const ParquetTables::ArrowTable& S) {
  const auto suppkey = int_values(column(L, "l_suppkey"));
  const auto s_key = int_values(column(S, "s_suppkey"));
  const auto s_nation = int_values(column(S, "s_nationkey"));
  int32_t max_suppkey = -1;
  for (int32_t k : s_key) max_suppkey = std::max(max_suppkey, k);
  std::vector<int16_t> nation_by_key(max_suppkey >= 0 ? static_cast<size_t>(max_suppkey) + 1 : 0, int16_t(-1));
  for (size_t i = 0; i < s_key.size(); ++i)
    if (s_key[i] >= 0 && static_cast<size_t>(s_key[i]) < nation_by_key.size())
      nation_by_key[static_cast<size_t>(s_key[i])] = static_cast<int16_t>(s_nation[i]);
  std::vector<int16_t> out(suppkey.size(), int16_t(-1));
  for (size_t i = 0; i < suppkey.size(); ++i)
    if (suppkey[i] >= 0 && static_cast<size_t>(suppkey[i]) < nation_by_key.size())
      out[i] = nation_by_key[static_cast<size_t>(suppkey[i])];
  return out;
}

// Latest shipdate of each lineitem's builder shard (bespoke_tpch/builder_impl.cpp:855-911):
// shards group lineitems by (ship year-month, discount, quantity / 100,
// supplier nation).  Keys and buckets are formed by the builder's own expressions.
std::vector<int16_t> shard_max_shipdates(const LineitemHost& h, int32_t base_days) {
  const size_t n = h.ship.size();
  std::vector<int64_t> keys(n);
  std::unordered_map<int64_t, int16_t> shard_max;
  for (size_t i = 0; i < n; ++i) {
    int y = 0;
    unsigned m = 0, d = 0;
    civil_from_days(base_days + h.ship[i], y, m, d);
    const int16_t supp_nation = h.supp_nation[i];
    const int32_t discount_bucket = static_cast<int32_t>(h.d8[i]);
    const int32_t quantity_bucket = static_cast<int32_t>(h.q16[i]) / 100;
    const int32_t month_index = y * 12 + (static_cast<int32_t>(m) - 1);
    const uint8_t supp_bucket = static_cast<uint8_t>(supp_nation >= 0 ? supp_nation : 255);
    keys[i] = (static_cast<int64_t>(month_index) << 24) | (static_cast<int64_t>(discount_bucket) << 16) |
              (static_cast<int64_t>(quantity_bucket) << 8) | static_cast<int64_t>(supp_bucket);
    auto it = shard_max.find(keys[i]);
    if (it == shard_max.end())
      shard_max.emplace(keys[i], h.ship[i]);
    else
      it->second = std::max(it->second, h.ship[i]);
  }
  std::vector<int16_t> out(n);
  for (size_t i = 0; i < n; ++i) out[i] = shard_max.find(keys[i])->second;
  return out;
}

LineitemHost derive_lineitem(const ParquetTables::ArrowTable& L, const ParquetTables::ArrowTable& S,
                             int32_t base_days) {
  LineitemHost h;
  auto commit_receipt = std::async(std::launch::async, [&] {
    const auto commit = date_offsets(column(L, "l_commitdate"), base_days);
    const auto receipt = date_offsets(column(L, "l_receiptdate"), base_days);
    std::vector<uint32_t> packed(commit.size());  // builder_impl.cpp:534-544
    for (size_t i = 0; i < commit.size(); ++i)
      packed[i] = (static_cast<uint32_t>(static_cast<uint16_t>(receipt[i])) << 16) |
                  static_cast<uint32_t>(static_cast<uint16_t>(commit[i]));
    return packed;
  });
  auto supp_nation = std::async(std::launch::async, [&] { return supplier_nations(L, S); });
  auto shipmode = std::async(std::launch::async, [&] {
    Dictionary dict;
    auto codes = dictionary_codes(column(L, "l_shipmode"), dict);
    return std::make_pair(std::move(codes), std::move(dict));
  });
  auto shipinstruct = std::async(std::launch::async, [&] {
    Dictionary dict;
    auto codes = dictionary_codes(column(L, "l_shipinstruct"), dict);
    return std::make_pair(std::move(codes), std::move(dict));
  });
  auto price = std::async(std::launch::async, [&] { return scaled_values(column(L, "l_extendedprice"), kPriceScale); });
  auto discount = std::async(std::launch::async, [&] { return scaled_values(column(L, "l_discount"), kDiscountScale); });
  auto tax = std::async(std::launch::async, [&] { return scaled_values(column(L, "l_tax"), kDiscountScale); });
  auto quantity = std::async(std::launch::async, [&] { return scaled_values(column(L, "l_quantity"), kPriceScale); });
  auto ship = std::async(std::launch::async, [&] { return date_offsets(column(L, "l_shipdate"), base_days); });
  h.orderkey = int_values(column(L, "l_orderkey"));
  const auto rf = dictionary_codes(column(L, "l_returnflag"), h.returnflag);
  const auto ls = dictionary_codes(column(L, "l_linestatus"), h.linestatus);
  const size_t n = h.orderkey.size();
  const size_t ls_count = h.linestatus.values.size();
  if (h.returnflag.values.size() * ls_count > 255)
    throw std::runtime_error("Lineitem returnflag/linestatus exceeds uint8 capacity");
  h.price = price.get();
  const auto disc = discount.get();
  const auto tx = tax.get();
  const auto qty = quantity.get();
  h.ship = ship.get();
  h.d8.resize(n);
  h.t8.resize(n);
  h.code.resize(n);
  h.q16.resize(n);
  h.dprice.resize(n);
  for (size_t i = 0; i < n; ++i) {
    h.d8[i] = static_cast<uint8_t>(disc[i]);
    h.t8[i] = static_cast<uint8_t>(tx[i]);
    h.q16[i] = static_cast<int16_t>(qty[i]);
    h.dprice[i] = static_cast<int32_t>(static_cast<int64_t>(h.price[i]) * (kDiscountScale - static_cast<int32_t>(h.d8[i])) /
                                       kDiscountScale);
    h.code[i] = static_cast<uint8_t>(rf[i] * ls_count + ls[i]);
  }
  for (size_t i = 0; i < n; ++i) {  // builder_impl.cpp:569-577
    if (i > 0 && h.orderkey[i] < h.orderkey[i - 1]) h.orderkey_sorted = false;
    h.max_orderkey = std::max(h.max_orderkey, h.orderkey[i]);
  }
  h.partkey = int_values(column(L, "l_partkey"));
  h.suppkey = int_values(column(L, "l_suppkey"));
  h.supp_nation = supp_nation.get();
  h.commit_receipt = commit_receipt.get();
  auto sm = shipmode.get();
  h.shipmode = std::move(sm.first);
  h.shipmode_dict = std::move(sm.second);
  auto si = shipinstruct.get();
  h.shipinstruct = std::move(si.first);
  h.shipinstruct_dict = std::move(si.second);
  for (int32_t k : h.partkey) h.max_partkey = std::max(h.max_partkey, k);
  // Q12's shard pruning can only drop a lineitem received more than 30 days
  // after shipping; without one the per-shard maxima are not needed.
  bool late = false;
  for (size_t i = 0; i < n && !late; ++i)
    late = static_cast<int32_t>(static_cast<int16_t>(h.commit_receipt[i] >> 16)) - static_cast<int32_t>(h.ship[i]) > 30;
  if (late) h.shard_max_ship = shard_max_shipdates(h, base_days);
  return h;
}

// orders, stably sorted by orderdate, the orderkey -> row map and the comments
// in the same order (bespoke_tpch/builder_impl.cpp:350-371, 580-642).
OrdersHost derive_orders(const ParquetTables::ArrowTable& O, int32_t base_days) {
  OrdersHost h;
  auto comment_f = std::async(std::launch::async, [&] { return string_column(column(O, "o_comment")); });
  const auto okey = int_values(column(O, "o_orderkey"));
  const auto ckey = int_values(column(O, "o_custkey"));
  const auto odate = date_offsets(column(O, "o_orderdate"), base_days);
  const auto prio = int_values(column(O, "o_shippriority"));
  const auto total = scaled_values(column(O, "o_totalprice"), kPriceScale);
  const auto priority = dictionary_codes(column(O, "o_orderpriority"), h.priority_dict);
  const auto status = dictionary_codes(column(O, "o_orderstatus"), h.status_dict);
  std::vector<uint32_t> order(okey.size());
  std::iota(order.begin(), order.end(), 0u);
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return odate[a] < odate[b]; });
  h.okey = permute(okey, order);
  h.ckey = permute(ckey, order);
  h.prio = permute(prio, order);
  h.odate = permute(odate, order);
  h.total = permute(total, order);
  h.priority = permute(priority, order);
  h.status = permute(status, order);
  int32_t max_key = -1;
  for (int32_t k : h.okey) max_key = std::max(max_key, k);
  h.map.assign(max_key >= 0 ? static_cast<size_t>(max_key) + 1 : 0, -1);
  for (size_t i = 0; i < h.okey.size(); ++i)
    if (h.okey[i] >= 0 && static_cast<size_t>(h.okey[i]) < h.map.size()) h.map[static_cast<size_t>(h.okey[i])] = static_cast<int32_t>(i);
  const StringColumn comment = comment_f.get();
  h.comment_bytes.reserve(comment.data.size());
  h.comment_offsets.reserve(order.size() + 1);
  h.comment_offsets.push_back(0);
  for (const uint32_t i : order) {
    const auto v = comment.view(i);
    h.comment_bytes.insert(h.comment_bytes.end(), v.begin(), v.end());
    h.comment_offsets.push_back(static_cast<uint32_t>(h.comment_bytes.size()));
  }
  return h;
}

// customer: keys, market-segment codes, nationkeys, the custkey -> row map and
// the strings of result rows (bespoke_tpch/builder_impl.cpp:670-700).
CustomerHost derive_customer(const ParquetTables::ArrowTable& C) {
  CustomerHost h;
  auto strings = std::async(std::launch::async, [&] {
    return std::array<StringColumn, 4>{string_column(column(C, "c_name")), string_column(column(C, "c_address")),
                                       string_column(column(C, "c_phone")), string_column(column(C, "c_comment"))};
  });
  h.ckey = int_values(column(C, "c_custkey"));
  h.seg = dictionary_codes(column(C, "c_mktsegment"), h.mktsegment);
  h.nkey = int_values(column(C, "c_nationkey"));
  h.acctbal = scaled_values(column(C, "c_acctbal"), kPriceScale);
  for (int32_t k : h.ckey) h.max_key = std::max(h.max_key, k);
  h.map.assign(h.ckey.empty() ? 0 : static_cast<size_t>(h.max_key) + 1, -1);
  for (size_t i = 0; i < h.ckey.size(); ++i)
    if (h.ckey[i] >= 0) h.map[static_cast<size_t>(h.ckey[i])] = static_cast<int32_t>(i);
  auto s = strings.get();
  h.name = std::move(s[0]);
  h.address = std::move(s[1]);
  h.phone = std::move(s[2]);
  h.comment = std::move(s[3]);
  return h;
}

// Q14's partkey -> promo flag table (bespoke_tpch/query_q14.cpp:193-223):
// types starting with "PROMO" by dictionary code, then each part row's key
// (non-negative keys; a later row with the same key wins).
struct PartHost {
  std::vector<int8_t> promo_by_key;
  int32_t max_key = -1;
  std::vector<int32_t> key, size, row_by_key;
  StringColumn name;
  std::vector<uint16_t> brand, container, type, mfgr;
  Dictionary brand_dict, container_dict, type_dict, mfgr_dict;
};

PartHost derive_part(const ParquetTables::ArrowTable& P) {
  PartHost h;
  h.key = int_values(column(P, "p_partkey"));
  h.name = string_column(column(P, "p_name"));
  h.size = int_values(column(P, "p_size"));
  const auto& key = h.key;
  h.brand = dictionary_codes(column(P, "p_brand"), h.brand_dict);
  h.mfgr = dictionary_codes(column(P, "p_mfgr"), h.mfgr_dict);
  h.container = dictionary_codes(column(P, "p_container"), h.container_dict);
  h.type = dictionary_codes(column(P, "p_type"), h.type_dict);
  const auto& type = h.type;
  const Dictionary& types = h.type_dict;
  if (key.empty()) return h;
  h.max_key = *std::max_element(key.begin(), key.end());
  if (h.max_key < 0) return h;
  std::vector<int8_t> promo_type(types.values.size(), 0);
  for (size_t c = 0; c < types.values.size(); ++c)
    promo_type[c] = types.values[c].size() >= 5 && types.values[c].compare(0, 5, "PROMO") == 0 ? 1 : 0;
  h.promo_by_key.assign(static_cast<size_t>(h.max_key) + 1, int8_t(-1));
  for (size_t i = 0; i < key.size(); ++i)
    if (key[i] >= 0) h.promo_by_key[static_cast<size_t>(key[i])] = promo_type[type[i]];
  h.row_by_key.assign(static_cast<size_t>(h.max_key) + 1, -1);  // the last row of a key (query_q19.cpp:242)
  for (size_t i = 0; i < key.size(); ++i)
    if (key[i] >= 0) h.row_by_key[static_cast<size_t>(key[i])] = static_cast<int32_t>(i);
  return h;
}

}  // namespace

Database* build(ParquetTables* tables) {
  const auto t0 = std::chrono::steady_clock::now();
  // A query's result rows are one std::vector of a few MB (Q10: ~100 bytes per
  // customer of the result).  Above glibc's default mmap threshold each such
  // vector is a fresh mapping, so every query would pay a page fault per 4 KB
  // of rows (0.8 ms of Q10's 1.1 ms at 38k rows); kept on the heap below 256 MB
  // and not trimmed, they reuse pages already faulted in by earlier queries.
  mallopt(M_MMAP_THRESHOLD, 256 << 20);
  mallopt(M_TRIM_THRESHOLD, 1 << 30);
  // BO_BUILD_TRACE set: the phases' end times (ms since build() began) on stderr.
  const bool trace = std::getenv("BO_BUILD_TRACE") != nullptr;
  auto phase = [&](const char* name) {
    if (trace)
      std::cerr << "build " << name << " ms: "
                << std::chrono::duration_cast<std::chrono::microseconds>(std::chrono::steady_clock::now() - t0).count() /
                       1000.0
                << "\n";
  };
  const int32_t base_days = static_cast<int32_t>(days_from_civil(1992, 1, 1));
  // Each table's host derivations on its own thread (as the reference's
  // builder runs one std::async task per table), overlapped with the
  // device context's creation.
  auto lineitem_f = std::async(std::launch::async, [&] { return derive_lineitem(tables->lineitem, tables->supplier, base_days); });
  auto orders_f = std::async(std::launch::async, [&] { return derive_orders(tables->orders, base_days); });
  auto customer_f = std::async(std::launch::async, [&] { return derive_customer(tables->customer); });
  auto part_f = std::async(std::launch::async, [&] { return derive_part(tables->part); });
  auto* db = new Database();
  db->base_date_days = base_days;
  await_device_init();
  const int rc = bo_create(&db->ctx, device_from_env());
  if (rc != BO_OK) {
    delete db;
    throw std::runtime_error("bo_create failed (status " + std::to_string(rc) + "): an sm_100 GPU is required");
  }
  phase("context");
  bo_ctx* ctx = db->ctx;
  try {
    {
      LineitemHost h = lineitem_f.get();
      phase("lineitem derived");
      db->returnflag = std::move(h.returnflag);
      db->linestatus = std::move(h.linestatus);
      db->n_lineitem = static_cast<int64_t>(h.orderkey.size());
      db->lineitem_orderkey_sorted = h.orderkey_sorted;
      db->max_lineitem_orderkey = h.max_orderkey;
      db->l_orderkey = upload(ctx, h.orderkey);
      db->l_shipdate = upload(ctx, h.ship);
      db->l_returnflag_linestatus = upload(ctx, h.code);
      db->l_extendedprice = upload(ctx, h.price);
      db->l_discounted_price = upload(ctx, h.dprice);
      db->l_discount = upload(ctx, h.d8);
      db->l_tax = upload(ctx, h.t8);
      db->l_quantity = upload(ctx, h.q16);
      db->shipmode = std::move(h.shipmode_dict);
      db->l_shipmode = upload(ctx, h.shipmode);
      db->l_commit_receipt = upload(ctx, h.commit_receipt);
      if (!h.shard_max_ship.empty()) db->l_shard_max_shipdate = upload(ctx, h.shard_max_ship);
      db->l_partkey = upload(ctx, h.partkey);
      db->l_supp_nation = upload(ctx, h.supp_nation);
      db->l_suppkey = upload(ctx, h.suppkey);
      db->shipinstruct = std::move(h.shipinstruct_dict);
      db->l_shipinstruct = upload(ctx, h.shipinstruct);
      db->max_lineitem_partkey = h.max_partkey;
      phase("lineitem uploaded");
    }
    std::vector<int32_t> order_custkeys;  // date-sorted orders' custkeys, for orders.cust_nationkey
    {
      OrdersHost h = orders_f.get();
      phase("orders derived");
      db->n_orders = static_cast<int64_t>(h.okey.size());
      db->n_orderkey_map = static_cast<int64_t>(h.map.size());
      if (!h.odate.empty()) {  // date-sorted: the first and last rows
        db->o_min_date = h.odate.front();
        db->o_max_date = h.odate.back();
      }
      check(ctx, bo_device_alloc(ctx, std::max<size_t>(h.map.size(), 256), &db->o_year_by_key.ptr), "device alloc");
      db->o_year_by_key.rows = db->n_orderkey_map;
      db->o_orderkey = upload(ctx, h.okey);
      db->o_custkey = upload(ctx, h.ckey);
      db->o_orderdate = upload(ctx, h.odate);
      db->o_shippriority = upload(ctx, h.prio);
      db->o_totalprice = upload(ctx, h.total);
      db->orderpriority = std::move(h.priority_dict);
      db->o_orderpriority = upload(ctx, h.priority);
      db->orderstatus = std::move(h.status_dict);
      db->o_orderstatus = upload(ctx, h.status);
      db->orderkey_to_row = upload(ctx, h.map);
      db->dense_orderkeys = !h.okey.empty() && h.okey.front() == 1 && h.okey.back() == static_cast<int32_t>(h.okey.size());
      db->o_comment = upload(ctx, h.comment_bytes);
      db->o_comment_offsets = upload(ctx, h.comment_offsets);
      // Per-order lineitem ranges (builder_impl.cpp:930-990), built on the device.
      const size_t bytes = std::max<size_t>(4 * h.okey.size(), 256);
      check(ctx, bo_device_alloc(ctx, bytes, &db->o_li_begin.ptr), "device alloc");
      check(ctx, bo_device_alloc(ctx, bytes, &db->o_li_end.ptr), "device alloc");
      db->o_li_begin.rows = db->o_li_end.rows = db->n_orders;
      order_custkeys = std::move(h.ckey);
      check(ctx,
            bo_tpch_order_ranges(ctx, col<int32_t>(db->l_orderkey), db->n_lineitem, col<int32_t>(db->orderkey_to_row),
                                 db->n_orderkey_map, db->n_orders, static_cast<uint32_t*>(db->o_li_begin.ptr),
                                 static_cast<uint32_t*>(db->o_li_end.ptr)),
            "order ranges");
      phase("orders uploaded");
    }
    {
      CustomerHost h = customer_f.get();
      phase("customer derived");
      db->n_customer = static_cast<int64_t>(h.ckey.size());
      db->custkey_bound = h.ckey.empty() ? 0 : h.max_key + 1;
      db->dense_custkeys = !h.ckey.empty() && h.ckey.front() == 1 && h.ckey.back() == static_cast<int32_t>(h.ckey.size());
      db->n_custkey_map = static_cast<int64_t>(h.map.size());
      db->mktsegment = std::move(h.mktsegment);
      db->c_custkey = upload(ctx, h.ckey);
      db->c_mktsegment = upload(ctx, h.seg);
      db->c_nationkey = upload(ctx, h.nkey);
      db->custkey_to_row = upload(ctx, h.map);
      // Each order's customer nation (builder_impl.cpp:672-690, 913-928): the
      // nationkey (as int16) of the last customer row of its custkey, -1 without one.
      std::vector<int16_t> nation_by_custkey(h.ckey.empty() || h.max_key < 0 ? 0 : static_cast<size_t>(h.max_key) + 1,
                                             int16_t(-1));
      for (size_t i = 0; i < h.ckey.size(); ++i)
        if (h.ckey[i] >= 0 && static_cast<size_t>(h.ckey[i]) < nation_by_custkey.size())
          nation_by_custkey[static_cast<size_t>(h.ckey[i])] = static_cast<int16_t>(h.nkey[i]);
      std::vector<int16_t> cust_nation(order_custkeys.size(), int16_t(-1));
      for (size_t i = 0; i < order_custkeys.size(); ++i)
        if (order_custkeys[i] >= 0 && static_cast<size_t>(order_custkeys[i]) < nation_by_custkey.size())
          cust_nation[i] = nation_by_custkey[static_cast<size_t>(order_custkeys[i])];
      db->o_cust_nation = upload(ctx, cust_nation);
      // Q22's per-custkey order bits (the builder's orders-by-customer
      // offsets, builder_impl.cpp:625-660: custkeys 0 .. largest order custkey).
      int32_t max_order_custkey = -1;
      for (int32_t k : order_custkeys) max_order_custkey = std::max(max_order_custkey, k);
      db->n_order_custkeys = max_order_custkey >= 0 ? static_cast<int64_t>(max_order_custkey) + 1 : 0;
      std::vector<uint32_t> has_order(static_cast<size_t>((db->n_order_custkeys + 31) / 32), 0u);
      for (int32_t k : order_custkeys)
        if (k >= 0) has_order[static_cast<size_t>(k) >> 5] |= 1u << (k & 31);
      db->o_has_order = upload(ctx, has_order);
      // Phone classes (builder_impl.cpp:152-178; query_q22.cpp:120-140).
      std::vector<uint8_t> prefix(h.ckey.size(), uint8_t(255));
      std::vector<uint32_t> pair(h.ckey.size(), 0u);
      for (size_t i = 0; i < h.ckey.size() && i + 1 < h.phone.offsets.size(); ++i) {
        const auto v = h.phone.view(i);
        if (v.size() < 2) continue;
        const char c0 = v[0], c1 = v[1];
        if (c0 >= '0' && c0 <= '9' && c1 >= '0' && c1 <= '9') prefix[i] = static_cast<uint8_t>((c0 - '0') * 10 + (c1 - '0'));
        pair[i] = 0x10000u | (static_cast<uint32_t>(static_cast<uint8_t>(c0)) << 8) | static_cast<uint8_t>(c1);
      }
      db->c_phone_prefix = upload(ctx, prefix);
      db->c_phone_pair = upload(ctx, pair);
      db->c_acctbal_device = upload(ctx, h.acctbal);
      db->c_name_offsets = upload(ctx, h.name.offsets);
      db->c_address_offsets = upload(ctx, h.address.offsets);
      db->c_phone_offsets = upload(ctx, h.phone.offsets);
      db->c_comment_offsets = upload(ctx, h.comment.offsets);
      db->c_acctbal = std::move(h.acctbal);
      db->c_name = std::move(h.name);
      db->c_address = std::move(h.address);
      db->c_phone = std::move(h.phone);
      db->c_comment = std::move(h.comment);
      phase("customer uploaded");
    }
    {
      PartHost h = part_f.get();
      db->max_partkey = h.max_key;
      db->n_promo_map = static_cast<int64_t>(h.promo_by_key.size());
      db->p_promo_by_key = upload(ctx, h.promo_by_key);
      db->n_part = static_cast<int64_t>(h.key.size());
      db->p_partkey = upload(ctx, h.key);
      db->p_brand = upload(ctx, h.brand);
      db->p_container = upload(ctx, h.container);
      db->brand = std::move(h.brand_dict);
      db->container = std::move(h.container_dict);
      db->p_type = upload(ctx, h.type);
      db->p_mfgr = upload(ctx, h.mfgr);
      db->mfgr = std::move(h.mfgr_dict);
      db->part_type = std::move(h.type_dict);
      db->p_name = upload(ctx, std::vector<char>(h.name.data.begin(), h.name.data.end()));
      db->p_name_offsets = upload(ctx, h.name.offsets);
      db->p_size = upload(ctx, h.size);
      db->p_row_by_key = upload(ctx, h.row_by_key);
    }
    // nation names by key (bespoke_tpch/builder_impl.cpp:780-803; query_q10.cpp:497-515)
    {
      const auto& N = tables->nation;
      const auto key = int_values(column(N, "n_nationkey"));
      const auto name = string_column(column(N, "n_name"));
      int32_t max_key = 0;
      for (int32_t k : key) max_key = std::max(max_key, k);
      db->nation_bound = max_key + 1;
      db->nation_name.assign(static_cast<size_t>(db->nation_bound), std::string());
      for (size_t i = 0; i < key.size(); ++i)
        if (key[i] >= 0) db->nation_name[static_cast<size_t>(key[i])] = std::string(name.view(i));
      for (const auto& nm : db->nation_name) db->nation_name_str.push_back(bo_host_str{nm.data(), nm.size()});
      db->nation_key = key;
      db->nation_regionkey = int_values(column(N, "n_regionkey"));
      for (size_t i = 0; i < key.size(); ++i) db->nation_row_name.emplace_back(name.view(i));
    }
    {  // partsupp (bespoke_tpch/builder_impl.cpp:751-777): value = supplycost * availqty, rows by partkey
      const auto& PS = tables->partsupp;
      const auto pk = int_values(column(PS, "ps_partkey"));
      const auto sk = int_values(column(PS, "ps_suppkey"));
      const auto qty = int_values(column(PS, "ps_availqty"));
      const auto cost = scaled_values(column(PS, "ps_supplycost"), kPriceScale);
      std::vector<uint32_t> order(pk.size());
      std::iota(order.begin(), order.end(), 0u);
      std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return pk[a] < pk[b]; });
      std::vector<int32_t> spk(pk.size()), ssk(pk.size()), val(pk.size()), scost(pk.size()), sqty(pk.size());
      for (size_t i = 0; i < order.size(); ++i) {
        spk[i] = pk[order[i]];
        ssk[i] = sk[order[i]];
        scost[i] = cost[order[i]];
        sqty[i] = qty[order[i]];
        val[i] = static_cast<int32_t>(static_cast<int64_t>(cost[order[i]]) * qty[order[i]]);
      }
      // Q9's part slots (query_q9.cpp:140-186): keys 0 .. the largest part or
      // partsupp key (0 without keys), each key's rows in this order.
      int32_t max_part_key = 0;
      for (int32_t k : spk) max_part_key = std::max(max_part_key, k);
      if (db->max_partkey > max_part_key) max_part_key = db->max_partkey;
      std::vector<int32_t> begin(static_cast<size_t>(max_part_key) + 2, 0);
      int32_t slots = 0;
      {
        size_t r = 0;
        while (r < spk.size() && spk[r] < 0) ++r;  // negative keys have no slot
        for (int64_t k = 0; k <= max_part_key; ++k) {
          begin[static_cast<size_t>(k)] = static_cast<int32_t>(r);
          const size_t r0 = r;
          while (r < spk.size() && spk[r] == k) ++r;
          slots = std::max(slots, static_cast<int32_t>(r - r0));
        }
        begin[static_cast<size_t>(max_part_key) + 1] = static_cast<int32_t>(r);
      }
      db->n_ps_part_keys = static_cast<int64_t>(max_part_key) + 1;
      db->ps_slots_per_part = std::max(slots, 1);
      db->ps_supplycost = upload(ctx, scost);
      db->ps_part_begin = upload(ctx, begin);
      db->n_partsupp = static_cast<int64_t>(pk.size());
      if (!spk.empty()) {
        db->ps_min_partkey = spk.front();
        db->ps_max_partkey = spk.back();
      }
      db->ps_partkey = upload(ctx, spk);
      db->ps_suppkey = upload(ctx, ssk);
      db->ps_value = upload(ctx, val);
      db->ps_availqty = upload(ctx, sqty);
    }
    {
      const auto& S = tables->supplier;
      db->s_suppkey = int_values(column(S, "s_suppkey"));
      db->s_nationkey = int_values(column(S, "s_nationkey"));
      db->s_name = string_column(column(S, "s_name"));
      db->s_address = string_column(column(S, "s_address"));
      db->s_phone = string_column(column(S, "s_phone"));
      db->s_comment = string_column(column(S, "s_comment"));
      // run_q16's supplier scan (query_q16.cpp:348-368): flags by suppkey over
      // keys 0 .. max(row count, largest key).
      int64_t bound = static_cast<int64_t>(db->s_suppkey.size());
      for (int32_t k : db->s_suppkey) bound = std::max<int64_t>(bound, k);
      db->n_s_banned = db->s_suppkey.empty() ? 0 : bound + 1;
      if (db->n_s_banned > 0) {
        db->s_comment_chars =
            upload(ctx, std::vector<char>(db->s_comment.data.begin(), db->s_comment.data.end()));
        db->s_comment_offsets = upload(ctx, db->s_comment.offsets);
        db->s_suppkey_device = upload(ctx, db->s_suppkey);
        check(ctx, bo_device_alloc(ctx, static_cast<size_t>(db->n_s_banned), &db->s_banned.ptr), "supplier flags");
        db->s_banned.rows = db->n_s_banned;
        check(ctx,
              bo_tpch_supplier_complaints(ctx, static_cast<const char*>(db->s_comment_chars.ptr),
                                          static_cast<const uint32_t*>(db->s_comment_offsets.ptr),
                                          static_cast<const int32_t*>(db->s_suppkey_device.ptr),
                                          static_cast<int64_t>(db->s_suppkey.size()),
                                          static_cast<uint8_t*>(db->s_banned.ptr), db->n_s_banned),
              "supplier flags");
      }
    }
    {  // Q20 and Q2 supplier derivations (query_q20.cpp:566-644, query_q2.cpp:167-212, 386-401)
      const auto& S = tables->supplier;
      const size_t ns = db->s_suppkey.size();
      db->s_acctbal = scaled_values(column(S, "s_acctbal"), kPriceScale);
      for (int32_t k : db->s_suppkey) db->s_max_suppkey = std::max(db->s_max_suppkey, k);
      // nationkey by suppkey, the last row of a key winning (builder_impl.cpp:725-742)
      std::vector<int16_t> by_key(db->s_max_suppkey >= 0 ? static_cast<size_t>(db->s_max_suppkey) + 1 : 0, int16_t(-1));
      for (size_t i = 0; i < ns; ++i)
        if (db->s_suppkey[i] >= 0) by_key[static_cast<size_t>(db->s_suppkey[i])] = static_cast<int16_t>(db->s_nationkey[i]);
      if (!by_key.empty()) db->s_nation_by_key = upload(ctx, by_key);
      // rows in s_name order
      std::vector<int32_t> by_name(ns);
      std::iota(by_name.begin(), by_name.end(), 0);
      std::stable_sort(by_name.begin(), by_name.end(),
                       [&](int32_t a, int32_t b) { return db->s_name.view(a) < db->s_name.view(b); });
      // run_q2's nation names by key, for keys below the nation row count (last row wins)
      const size_t n_nation = db->nation_key.size();
      db->nation_name_by_idx.assign(n_nation, std::string());
      for (size_t i = 0; i < n_nation; ++i)
        if (db->nation_key[i] >= 0 && static_cast<size_t>(db->nation_key[i]) < n_nation)
          db->nation_name_by_idx[static_cast<size_t>(db->nation_key[i])] = db->nation_row_name[i];
      db->s_nation_idx.assign(ns, -1);
      for (size_t i = 0; i < ns; ++i)
        if (static_cast<uint32_t>(db->s_nationkey[i]) < n_nation) db->s_nation_idx[i] = db->s_nationkey[i];
      auto nation_of = [&](size_t row) -> std::string_view {
        const int32_t idx = db->s_nation_idx[row];
        return idx >= 0 ? std::string_view(db->nation_name_by_idx[static_cast<size_t>(idx)]) : std::string_view();
      };
      std::vector<int32_t> order(ns);
      std::iota(order.begin(), order.end(), 0);
      std::sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
        if (db->s_acctbal[a] != db->s_acctbal[b]) return db->s_acctbal[a] > db->s_acctbal[b];
        const auto na = nation_of(a), nb = nation_of(b);
        if (na != nb) return na < nb;
        const auto sa = db->s_name.view(a), sb = db->s_name.view(b);
        if (sa != sb) return sa < sb;
        return a < b;
      });
      std::vector<uint32_t> rank(ns);
      for (size_t i = 0; i < ns; ++i) rank[static_cast<size_t>(order[i])] = static_cast<uint32_t>(i);
      if (ns > 0) {
        db->s_nationkey_device = upload(ctx, db->s_nationkey);
        db->s_row_by_name = upload(ctx, by_name);
        db->s_nation_idx_device = upload(ctx, db->s_nation_idx);
        db->s_rank = upload(ctx, rank);
      }
    }
    {  // brand and type ranks in string order (query_q16.cpp:491-512)
      auto ranks = [](const std::vector<std::string>& dict) {
        std::vector<uint32_t> idx(dict.size());
        std::iota(idx.begin(), idx.end(), 0u);
        std::sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) { return dict[a] < dict[b]; });
        std::vector<uint16_t> rank(dict.size());
        for (size_t i = 0; i < idx.size(); ++i) rank[idx[i]] = static_cast<uint16_t>(i);
        return rank;
      };
      if (db->brand.values.size() <= 65536) db->brand_rank = ranks(db->brand.values);
      if (db->part_type.values.size() <= 65536) db->type_rank = ranks(db->part_type.values);
    }
    {  // region name -> key, the first row of a name (builder_impl.cpp:805-826)
      const auto& R = tables->region;
      const auto key = int_values(column(R, "r_regionkey"));
      const auto name = string_column(column(R, "r_name"));
      for (size_t i = 0; i < key.size(); ++i) db->region_key_by_name.emplace(std::string(name.view(i)), key[i]);
    }
    check(ctx, bo_device_alloc(ctx, sizeof(bo_q1_agg) * BO_Q1_MAX_GROUPS + 256, &db->scratch.ptr), "scratch alloc");
    check(ctx, bo_synchronize(ctx), "build");
  } catch (...) {
    delete db;
    throw;
  }
  phase("done");
  const auto ms = std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::steady_clock::now() - t0).count();
  std::cout << "Build ms: " << ms << "\n";
  return db;
}

void query(Database* db) {
  struct Request {
    std::string id, line;
  };
  std::vector<Request> requests;
  std::string line;
  while (std::getline(std::cin, line)) {
    if (line.empty()) break;
    std::istringstream iss(line);
    std::string id = "0";
    iss >> id;
    if (!iss) continue;
    requests.push_back(Request{id, line});
  }
  // BO_EXEC_US set: each request also reports its time in microseconds on
  // stderr ("<idx> | Execution us: <us>"); stdout keeps the reference's lines.
  const bool exec_us = std::getenv("BO_EXEC_US") != nullptr;
  for (size_t idx = 0; idx < requests.size(); ++idx) {
    const auto& r = requests[idx];
    const auto start = std::chrono::steady_clock::now();
    auto report = [&](std::chrono::steady_clock::time_point end) {
      std::cout << (idx + 1) << " | Execution ms: "
                << std::chrono::duration_cast<std::chrono::milliseconds>(end - start).count() << "\n";
      if (exec_us)
        std::cerr << (idx + 1) << " | Execution us: "
                  << std::chrono::duration_cast<std::chrono::microseconds>(end - start).count() << "\n";
    };
    const std::string file = "result" + std::to_string(idx + 1) + ".csv";
    std::istringstream iss(r.line);
    std::string qid;
    iss >> qid;
    auto arg = [&](const char* name) {
      std::string v;
      if (!(iss >> std::quoted(v))) throw std::runtime_error("Q" + r.id + ": failed to parse " + name);
      return v;
    };
    if (r.id == "1") {
      const std::string delta = arg("DELTA");
      const auto rows = run_q1(*db, delta);
      const auto end = std::chrono::steady_clock::now();
      write_q1_csv(file, rows);
      report(end);
    } else if (r.id == "3") {
      const std::string segment = arg("SEGMENT");
      const std::string date = arg("DATE");
      const auto rows = run_q3(*db, segment, date);
      const auto end = std::chrono::steady_clock::now();
      write_q3_csv(*db, file, rows);
      report(end);
    } else if (r.id == "10") {
      const std::string date = arg("DATE");
      const auto rows = run_q10(*db, date);
      const auto end = std::chrono::steady_clock::now();
      write_q10_csv(file, rows);
      report(end);
    } else if (r.id == "4") {
      const std::string date = arg("DATE");
      const auto rows = run_q4(*db, date);
      const auto end = std::chrono::steady_clock::now();
      write_q4_csv(file, rows);
      report(end);
    } else if (r.id == "5") {
      const std::string region = arg("REGION");
      const std::string date = arg("DATE");
      const auto rows = run_q5(*db, region, date);
      const auto end = std::chrono::steady_clock::now();
      write_q5_csv(file, rows);
      report(end);
    } else if (r.id == "7") {
      const std::string nation1 = arg("NATION1");
      const std::string nation2 = arg("NATION2");
      const auto rows = run_q7(*db, nation1, nation2);
      const auto end = std::chrono::steady_clock::now();
      write_q7_csv(file, rows);
      report(end);
    } else if (r.id == "8") {
      const std::string nation = arg("NATION");
      const std::string region = arg("REGION");
      const std::string type = arg("TYPE");
      const auto rows = run_q8(*db, nation, region, type);
      const auto end = std::chrono::steady_clock::now();
      write_q8_csv(file, rows);
      report(end);
    } else if (r.id == "22") {
      std::vector<std::string> codes;
      for (const char* name : {"I1", "I2", "I3", "I4", "I5", "I6", "I7"}) codes.push_back(arg(name));
      const auto rows = run_q22(*db, codes);
      const auto end = std::chrono::steady_clock::now();
      write_q22_csv(file, rows);
      report(end);
    } else if (r.id == "11") {
      const std::string nation = arg("NATION");
      const std::string fraction = arg("FRACTION");
      const auto rows = run_q11(*db, nation, fraction);
      const auto end = std::chrono::steady_clock::now();
      write_q11_csv(file, rows);
      report(end);
    } else if (r.id == "15") {
      const std::string date = arg("DATE");
      arg("STREAM_ID");  // parsed as the reference does; not used by the query
      const auto rows = run_q15(*db, date);
      const auto end = std::chrono::steady_clock::now();
      write_q15_csv(file, rows);
      report(end);
    } else if (r.id == "9") {
      const std::string color = arg("COLOR");
      const auto rows = run_q9(*db, color);
      const auto end = std::chrono::steady_clock::now();
      write_q9_csv(file, rows);
      report(end);
    } else if (r.id == "21") {
      const std::string nation = arg("NATION");
      const auto rows = run_q21(*db, nation);
      const auto end = std::chrono::steady_clock::now();
      write_q21_csv(file, rows);
      report(end);
    } else if (r.id == "19") {
      std::string quantity[3], brand[3];
      for (int g = 0; g < 3; ++g) quantity[g] = arg(("QUANTITY" + std::to_string(g + 1)).c_str());
      for (int g = 0; g < 3; ++g) brand[g] = arg(("BRAND" + std::to_string(g + 1)).c_str());
      const auto rows = run_q19(*db, quantity, brand);
      const auto end = std::chrono::steady_clock::now();
      write_q19_csv(file, rows);
      report(end);
    } else if (r.id == "17") {
      const std::string brand = arg("BRAND");
      const std::string container = arg("CONTAINER");
      const auto rows = run_q17(*db, brand, container);
      const auto end = std::chrono::steady_clock::now();
      write_q17_csv(file, rows);
      report(end);
    } else if (r.id == "14") {
      const std::string date = arg("DATE");
      const auto rows = run_q14(*db, date);
      const auto end = std::chrono::steady_clock::now();
      write_q14_csv(file, rows);
      report(end);
    } else if (r.id == "12") {
      const std::string mode1 = arg("SHIPMODE1");
      const std::string mode2 = arg("SHIPMODE2");
      const std::string date = arg("DATE");
      const auto rows = run_q12(*db, mode1, mode2, date);
      const auto end = std::chrono::steady_clock::now();
      write_q12_csv(file, rows);
      report(end);
    } else if (r.id == "13") {
      const std::string word1 = arg("WORD1");
      const std::string word2 = arg("WORD2");
      const auto rows = run_q13(*db, word1, word2);
      const auto end = std::chrono::steady_clock::now();
      write_q13_csv(file, rows);
      report(end);
    } else if (r.id == "18") {
      const std::string quantity = arg("QUANTITY");
      const auto rows = run_q18(*db, quantity);
      const auto end = std::chrono::steady_clock::now();
      write_q18_csv(*db, file, rows);
      report(end);
    } else if (r.id == "20") {
      const std::string color = arg("COLOR");
      const std::string date = arg("DATE");
      const std::string nation = arg("NATION");
      const auto rows = run_q20(*db, color, date, nation);
      const auto end = std::chrono::steady_clock::now();
      write_q20_csv(file, rows);
      report(end);
    } else if (r.id == "2") {
      const std::string size = arg("SIZE");
      const std::string type = arg("TYPE");
      const std::string region = arg("REGION");
      const auto rows = run_q2(*db, size, type, region);
      const auto end = std::chrono::steady_clock::now();
      write_q2_csv(file, rows);
      report(end);
    } else if (r.id == "16") {
      const std::string brand = arg("BRAND");
      const std::string type = arg("TYPE");
      std::string sizes[8];
      static const char* const kSizeNames[8] = {"SIZE1", "SIZE2", "SIZE3", "SIZE4",
                                                "SIZE5", "SIZE6", "SIZE7", "SIZE8"};
      for (int i = 0; i < 8; ++i) sizes[i] = arg(kSizeNames[i]);
      const auto rows = run_q16(*db, brand, type, sizes);
      const auto end = std::chrono::steady_clock::now();
      write_q16_csv(file, rows);
      report(end);
    } else if (r.id == "6") {
      const std::string date = arg("DATE");
      const std::string discount = arg("DISCOUNT");
      const std::string quantity = arg("QUANTITY");
      const auto rows = run_q6(*db, date, discount, quantity);
      const auto end = std::chrono::steady_clock::now();
      write_q6_csv(file, rows);
      report(end);
    } else {
      // Not on the GPU path: the reference's stub record.
      std::ofstream out(file);
      out << "query_id,params\n" << escape_csv(r.id) << "," << escape_csv(r.line) << "\n";
      const auto end = std::chrono::steady_clock::now();
      report(end);
    }
  }
}
