"""The drop-in tests' Parquet writer (bespokeolap_artifacts_b200.tpch_data)."""
from bespokeolap_artifacts_b200.tpch_data import (  # noqa: F401
    BRANDS, COLORS, CONTAINERS, PART_TYPES, PRIORITIES, SEGMENTS, SHIPINSTRUCTS, SHIPMODES, WORDS,
    write_tpch)
