// ORACLE -- test infrastructure.  Declaration of the Parquet reader the
// reference's loader calls but does not ship (bespoke_tpch/loader_impl.cpp:3,12-19);
// defined in oracle/ref_harness.cpp with Arrow's Parquet reader.
#pragma once

#include <arrow/table.h>

#include <memory>
#include <string>

std::shared_ptr<arrow::Table> ReadParquetTable(const std::string& path);
