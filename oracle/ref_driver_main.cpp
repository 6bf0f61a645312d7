// ORACLE -- test infrastructure, not part of the product.
//
// Stand-in for the reference's external driver, linked with the reference's
// own loader_impl.cpp, builder_impl.cpp and query_impl.cpp compiled unchanged
// from the reference tree (recipe: oracle/build_oracle.py): load(argv[1]),
// build(), query() -- the same calls the GPU drop-in's driver makes, so the
// two produce result<idx>.csv files for the same requests that the tests
// compare.  Also defines the Parquet reader the reference's loader declares
// but does not ship (loader_utils.hpp).
#include <arrow/api.h>
#include <arrow/io/file.h>
#include <parquet/arrow/reader.h>

#include <iostream>
#include <memory>
#include <stdexcept>
#include <string>

#include "builder_impl.hpp"
#include "loader_impl.hpp"
#include "query_impl.hpp"

std::shared_ptr<arrow::Table> ReadParquetTable(const std::string& path) {
  auto file = arrow::io::ReadableFile::Open(path);
  if (!file.ok()) throw std::runtime_error("cannot open " + path);
  auto reader = parquet::arrow::OpenFile(*file, arrow::default_memory_pool());
  if (!reader.ok()) throw std::runtime_error("cannot read parquet " + path);
  auto table = (*reader)->ReadTable();
  if (!table.ok()) throw std::runtime_error("cannot read table " + path);
  return *table;
}

int main(int argc, char** argv) {
  if (argc < 2) {
    std::cerr << "usage: " << argv[0] << " <parquet dir prefix>\n";
    return 2;
  }
  ParquetTables* tables = load(argv[1]);
  Database* db = build(tables);
  query(db);
  return 0;
}
