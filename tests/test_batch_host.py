"""Host logic of the batching layer (no GPU): the autotuner's choice from
measured times, the tile table's round trip and size classes, and the C
layout of the batch structures."""
import ctypes as C
import shutil
import subprocess
from pathlib import Path

import pytest

from bespokeolap_artifacts_b200 import batching as B
from bespokeolap_artifacts_b200 import native as N

ROOT = Path(__file__).resolve().parent.parent


def fake_instances():
    return [B.Instance(N.BATCH_JOIN, 2_000_000, {}, {}), B.Instance(N.BATCH_JOIN, 3_000_000, {}, {}),
            B.Instance(N.BATCH_GROUPBY, 50_000, {}, {}), B.Instance(N.BATCH_SCAN_AGG, 70_000_000, {}, {})]


def test_size_bucket():
    assert B.size_bucket(0) == 4 and B.size_bucket(10_000) == 4 and B.size_bucket(99_999) == 4
    assert B.size_bucket(100_000) == 5 and B.size_bucket(60_000_000) == 7 and B.size_bucket(10**9) == 8


def test_autotune_picks_fastest_per_class():
    # Synthetic timer: joins like big tiles, group-bys like small ones, two
    # workers per SM are faster.
    def timer(engine, insts, workers, reps):
        t = sum((1e6 / i.tile_rows if i.kind == N.BATCH_JOIN else i.tile_rows / 1e4) for i in insts)
        return t * (0.5 if workers == 2 else 1.0)

    insts = fake_instances()
    table = B.autotune(None, insts, candidates=(32768, 131072, 524288), workers=(1, 2), timer=timer)
    assert table.tiles[str(N.BATCH_JOIN)][str(6)] == 524288
    assert table.tiles[str(N.BATCH_GROUPBY)][str(4)] == 32768
    assert table.workers_per_sm == 2
    assert [i.tile_rows for i in insts] == [524288, 524288, 32768, table.tile_for(N.BATCH_SCAN_AGG, 70_000_000)]
    again = B.TileTable.from_json(table.to_json())
    assert again.tiles == table.tiles and again.workers_per_sm == 2
    assert again.tile_for(N.BATCH_JOIN, 5_000_000) == 524288
    assert again.tile_for(N.BATCH_JOIN, 500) == B.DEFAULT_TILE  # unseen class -> default


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_batch_struct_layout_matches_header(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "bespoke_gpu.h"\n'
        'int main(void){printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(bo_batch_instance),'
        ' sizeof(bo_batch_result), offsetof(bo_batch_instance, fact), offsetof(bo_batch_instance, build),'
        ' offsetof(bo_batch_instance, a), offsetof(bo_batch_instance, categories),'
        ' offsetof(bo_batch_instance, n_categories), offsetof(bo_batch_result, join),'
        ' offsetof(bo_batch_result, groupby)); return 0;}\n')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", f"-I{ROOT / 'include'}", str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    want = [C.sizeof(N.BatchInstance), C.sizeof(N.BatchResult), N.BatchInstance.fact.offset,
            N.BatchInstance.build.offset, N.BatchInstance.a.offset, N.BatchInstance.categories.offset,
            N.BatchInstance.n_categories.offset, N.BatchResult.join.offset, N.BatchResult.groupby.offset]
    assert got == want


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_q3_struct_layout_matches_header(tmp_path):
    src = tmp_path / "q3layout.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "bespoke_gpu.h"\n'
        'int main(void){printf("%zu %zu %zu %zu %zu\\n", sizeof(bo_tpch_q3_tables), sizeof(bo_tpch_q3_row),'
        ' offsetof(bo_tpch_q3_tables, o_orderkey), offsetof(bo_tpch_q3_tables, l_orderkey),'
        ' offsetof(bo_tpch_q3_row, orderdate_offset)); return 0;}\n')
    exe = tmp_path / "q3layout"
    subprocess.run(["gcc", f"-I{ROOT / 'include'}", str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    want = [C.sizeof(N.TpchQ3Tables), C.sizeof(N.TpchQ3Row), N.TpchQ3Tables.o_orderkey.offset,
            N.TpchQ3Tables.l_orderkey.offset, N.TpchQ3Row.orderdate_offset.offset]
    assert got == want


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_q10_q18_struct_layouts_match_header(tmp_path):
    src = tmp_path / "q10layout.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "bespoke_gpu.h"\n'
        'int main(void){printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n",'
        ' sizeof(bo_tpch_q10_tables), sizeof(bo_tpch_q10_row), sizeof(bo_tpch_q18_tables), sizeof(bo_tpch_q18_row),'
        ' offsetof(bo_tpch_q10_tables, lineitem_orderkey_sorted), offsetof(bo_tpch_q10_tables, n_customer),'
        ' offsetof(bo_tpch_q10_row, nationkey), offsetof(bo_tpch_q18_tables, orderkey_bound),'
        ' offsetof(bo_tpch_q18_tables, dense_custkeys), offsetof(bo_tpch_q18_row, orderdate_offset)); return 0;}\n')
    exe = tmp_path / "q10layout"
    subprocess.run(["gcc", f"-I{ROOT / 'include'}", str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    want = [C.sizeof(N.TpchQ10Tables), C.sizeof(N.TpchQ10Row), C.sizeof(N.TpchQ18Tables), C.sizeof(N.TpchQ18Row),
            N.TpchQ10Tables.lineitem_orderkey_sorted.offset, N.TpchQ10Tables.n_customer.offset,
            N.TpchQ10Row.nationkey.offset, N.TpchQ18Tables.orderkey_bound.offset,
            N.TpchQ18Tables.dense_custkeys.offset, N.TpchQ18Row.orderdate_offset.offset]
    assert got == want
