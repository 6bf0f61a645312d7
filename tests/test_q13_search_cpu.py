"""The Q13 comment search's SWAR form (csrc/q13_search.cuh, shared by the
GPU kernel and this host build) against a byte-serial restatement of the
reference's find_substring / matches_pattern (bespoke_tpch/query_q13.cpp:
44-83): the fuzz program in tests/native is compiled with g++ and run.
CPU only."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_swar_search_matches_serial_search(tmp_path):
    exe = tmp_path / "q13_search_fuzz"
    subprocess.run(["g++", "-O2", "-std=c++17", f"-I{ROOT / 'bespokeolap_artifacts_b200' / 'csrc'}",
                    str(ROOT / "tests" / "native" / "q13_search_fuzz.cpp"), "-o", str(exe)], check=True)
    p = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    assert p.stdout.startswith("ok ")
