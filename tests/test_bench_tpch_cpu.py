"""bench.py's TPC-H section helpers on the CPU: every request of the
section is answered by the reference driver (compiled unchanged) on the
section's kind of seeded data, with one execution time per request and a
result file each.  The GPU driver's side runs in the bench itself."""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402
from tpch_parquet import write_tpch  # noqa: E402

REF_DRIVER = ROOT / "oracle" / "_ref" / "ref_tpch_driver"


@pytest.mark.skipif(not REF_DRIVER.exists(), reason="reference driver not built")
def test_section_requests_run_on_the_reference_driver(tmp_path):
    data = write_tpch(tmp_path / "d", n_customer=3000, n_orders=30000, seed=11, customer_nations="known",
                      n_supplier=200, n_part=4000, orderless_customers=True, lineitem_keys="partsupp")
    reqs = [r for _, r in bench.TPCH_REQUESTS]
    build_ms, times = bench._driver_times(REF_DRIVER, data, tmp_path / "ref", reqs, "ms")
    assert build_ms >= 0 and len(times) == len(reqs)
    for i in range(len(reqs)):
        lines = (tmp_path / "ref" / f"result{i + 1}.csv").read_text().splitlines()
        assert len(lines) >= 2, reqs[i]  # header and at least one row on this data
