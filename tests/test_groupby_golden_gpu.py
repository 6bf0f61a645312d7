"""The GPU group-by + top-k against answers the reference computed: run_q18's
dense aggregation of the same joined rows (tests/golden/make_golden_groupby.py,
fixtures in tests/golden/groupby_q18_reference.json).  Group count, joined
rows, and the top-10 a_ids with their counts in (count desc, a_id asc) order
must be equal, at the full A 2.5M / B 36M / C 4M size too, for every form the
engine runs: the plain exact-count pipeline, the presized one (under- and
over-predicted), the radix-partitioned one and the persistent batch kernel.
min(year) has no run_q18 counterpart; it is checked against the C
restatement in tests/test_groupby_gpu.py."""
import json
from pathlib import Path

import pytest

from bespokeolap_artifacts_b200 import batching as B
from bespokeolap_artifacts_b200 import native as N

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = json.loads((GOLDEN / "groupby_q18_reference.json").read_text())
K = 10


def golden_input(case):
    import sys

    if str(GOLDEN) not in sys.path:
        sys.path.insert(0, str(GOLDEN))
    import make_golden_groupby as MG

    g = MG.make_case(case["n_a"], case["n_b"], case["n_c"], case["seed"], case["variant"])
    assert MG.input_sha(g) == case["input_sha256"], "the seeded generator changed: regenerate the fixtures"
    g.k = K
    return g


def check(r, case):
    assert r["n_groups"] == case["n_groups"]
    assert r["joined_rows"] == case["joined_rows"]
    assert r["keys"] == case["keys"][:K]
    assert r["counts"] == case["counts"][:K]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"b{c['n_b']}-seed{c['seed']}-{c['variant']}")
def test_groupby_forms_match_reference_q18(engine, torch_cuda, case):
    torch = torch_cuda
    g = golden_input(case)
    dev = engine.groupby_to_device(g)
    check(engine.groupby_plain(dev, g), case)
    for scale in (0.3, 1.0, 3.0):  # an under-prediction reruns exactly
        pred = torch.tensor([max(case["n_groups"], 1) * scale], dtype=torch.float32, device="cuda")
        check(engine.groupby_presized(dev, g, pred), case)
    check(engine.groupby_partitioned(dev, g, 6, float(max(case["joined_rows"], 1))), case)
    inst = B.Instance(N.BATCH_GROUPBY, len(g.b_a), {k: dev[k] for k in ("a_ids", "b_a", "b_c", "c_cat", "c_year")},
                      dict(cat_set=[int(v) for v in g.cat_set], year_lo=g.year_lo, year_hi=g.year_hi, k=K,
                           a_id_max=dev["a_id_max"]))
    b = B.Batch(engine, [inst])
    try:
        check(b.run()[0], case)
    finally:
        b.close()
