"""The drop-in library exports the reference's three C++ entry points under
the reference's own (Itanium-mangled) names, so the reference's external
driver links against it unchanged (bespoke_tpch/loader_impl.hpp:20,
builder_impl.hpp:173, query_impl.hpp:6); and its loader reads the same file
names (bespoke_tpch/loader_impl.cpp:12-19)."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
LIB = ROOT / "bespokeolap_artifacts_b200" / "host" / "libbespoke_tpch_gpu.so"

ENTRY_POINTS = {
    "_Z4loadNSt7__cxx1112basic_stringIcSt11char_traitsIcESaIcEEE": "load(std::string)",
    "_Z5buildP13ParquetTables": "build(ParquetTables*)",
    "_Z5queryP8Database": "query(Database*)",
}


@pytest.mark.skipif(shutil.which("nm") is None, reason="needs nm")
def test_exports_reference_entry_points():
    if not LIB.exists():
        pytest.skip("drop-in library not built")
    out = subprocess.run(["nm", "-D", "--defined-only", str(LIB)], capture_output=True, text=True, check=True).stdout
    names = {line.split()[-1] for line in out.splitlines() if line.strip()}
    for sym, sig in ENTRY_POINTS.items():
        assert sym in names, sig


def test_loader_reads_the_reference_file_names():
    src = (ROOT / "bespokeolap_artifacts_b200" / "host" / "tpch_gpu.cpp").read_text()
    for t in ("customer", "lineitem", "nation", "orders", "part", "partsupp", "region", "supplier"):
        assert f'"{t}.parquet"' in src
