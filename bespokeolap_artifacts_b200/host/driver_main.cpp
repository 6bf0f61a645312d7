// Stand-in for the reference's external driver (bespoke-olap's runner links
// load / build / query and calls them in this order): the parquet directory
// prefix is the only argument, requests come on stdin.
#include <iostream>

#include "tpch_gpu.hpp"

int main(int argc, char** argv) {
  if (argc < 2) {
    std::cerr << "usage: " << argv[0] << " <parquet dir prefix, e.g. data/>\n";
    return 2;
  }
  ParquetTables* tables = load(argv[1]);
  Database* db = build(tables);
  query(db);
  delete db;
  delete tables;
  return 0;
}
