"""GPU parity of the scan / filter / group-aggregate kernels (Q1 and Q6 shapes)
against the oracle and the compiled reference.  Integer totals must be
bit-exact; the Q1 doubles, computed by run_q1's own expressions from those
integers, must be bitwise equal to the reference's."""
import ctypes as C

import numpy as np
import pytest

from bespokeolap_artifacts_b200 import datagen as dg
from bespokeolap_artifacts_b200 import native as N
from bespokeolap_artifacts_b200.engine import Q1ResultRow, q1_rows_from_aggs
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def to_dev(torch, arrs):
    return [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in arrs]


@pytest.mark.parametrize("n,seed", [(0, 1), (1, 2), (3, 3), (4, 4), (7, 5), (1023, 6), (65_537, 7), (1_000_003, 8)])
def test_q1_fact_host_matches_oracle(engine, n, seed):
    t = dg.gen_fact(n, seed)
    got = engine.q1_fact_host(t, dg.Q1_CUTOFF)
    want, rc = O.q1_fact(t, dg.Q1_CUTOFF)
    assert rc == 0
    assert got == want


@pytest.mark.parametrize("cutoff", [dg.DATE_LO - 1, dg.DATE_LO, 9000, dg.Q1_CUTOFF, dg.DATE_HI])
def test_q1_fact_cutoffs(engine, cutoff):
    t = dg.gen_fact(100_000, 9)
    assert engine.q1_fact_host(t, cutoff) == O.q1_fact(t, cutoff)[0]


def test_q1_fact_device_full_size(engine, torch_cuda):
    torch = torch_cuda
    t = dg.gen_fact(6_000_000, 10)
    cols = to_dev(torch, t.columns())
    out = torch.zeros(N.Q1_MAX_GROUPS * C.sizeof(N.Q1Agg), dtype=torch.uint8, device="cuda")
    for _ in range(2):  # accumulators must be left clean for the next call
        engine.q1_fact_device(cols, t.n_rows, dg.Q1_CUTOFF, 3, 2, out)
        engine.synchronize()
        host = out.cpu().numpy()
        aggs = (N.Q1Agg * 6).from_buffer_copy(host.tobytes()[: 6 * C.sizeof(N.Q1Agg)])
        assert [a.as_dict() for a in aggs] == O.q1_fact(t, dg.Q1_CUTOFF)[0]


def test_q1_fact_rows_bitwise_equal_reference(engine):
    if not O.ref_available():
        pytest.skip("compiled reference harness missing")
    t = dg.gen_fact(200_003, 11)
    db = O.RefDatabase(dg.fact_as_lineitem(t))
    ref, _ = db.q1(90)
    got = engine.run_q1_fact(t, 90)
    assert len(got) == len(ref)
    for g, r in zip(got, ref):
        for f in Q1ResultRow.__dataclass_fields__:
            assert getattr(g, f) == r[f], f


def test_q1_storage_layout_bitwise_equal_reference(engine):
    """The storage-plan kernel fed the columns the reference's own builder
    derived reproduces run_q1 exactly (same dictionaries, same doubles)."""
    if not O.ref_available():
        pytest.skip("compiled reference harness missing")
    t = dg.gen_fact(300_001, 12)
    db = O.RefDatabase(dg.fact_as_lineitem(t))
    li = db.lineitem()
    for delta in (90, 1, 2000):
        ref, _ = db.q1(delta)
        got = engine.run_q1(li, delta)
        assert [tuple(vars(g).values()) for g in got] == [
            tuple(r[f] for f in Q1ResultRow.__dataclass_fields__) for r in ref]


@pytest.mark.parametrize("n", [0, 5, 8, 9, 4096 + 3, 500_000])
def test_q1_storage_layout_matches_oracle(engine, n):

    t = dg.gen_fact(n, 13)
    li = dg.fact_to_storage_plan(t)
    cut = dg.Q1_CUTOFF - 8035
    assert engine.q1_lineitem_host(li, cut, 6) == O.q1_lineitem(li, cut, 6)[0]


def test_q1_bad_group_code_is_an_error(engine):
    t = dg.gen_fact(10_000, 14)
    t.flag_a[123] = 7  # outside the declared 3 x 2 domain
    t.ship_date[123] = dg.DATE_LO
    with pytest.raises(N.BoError) as e:
        engine.q1_fact_host(t, dg.Q1_CUTOFF)
    assert e.value.status == -6
    # the context stays usable and the accumulators clean
    t2 = dg.gen_fact(10_000, 15)
    assert engine.q1_fact_host(t2, dg.Q1_CUTOFF) == O.q1_fact(t2, dg.Q1_CUTOFF)[0]


def test_q1_value_out_of_contract_is_an_error(engine):
    t = dg.gen_fact(1000, 16)
    t.discount[5] = 250
    t.ship_date[5] = dg.DATE_LO
    with pytest.raises(N.BoError) as e:
        engine.q1_fact_host(t, dg.Q1_CUTOFF)
    assert e.value.status == -6


def test_q1_misaligned_pointer_rejected(engine, torch_cuda):
    torch = torch_cuda
    t = dg.gen_fact(1000, 17)
    cols = to_dev(torch, t.columns())
    buf = torch.zeros(4004, dtype=torch.uint8, device="cuda")
    cols[0] = buf[4:].view(torch.int32)  # 4-byte offset
    out = torch.zeros(8 * C.sizeof(N.Q1Agg), dtype=torch.uint8, device="cuda")
    with pytest.raises(N.BoError) as e:
        engine.q1_fact_device(cols, 1000, dg.Q1_CUTOFF, 3, 2, out)
    assert e.value.status == -1


@pytest.mark.parametrize("params", [(731, 1096, 5, 7, 2400), (0, 2557, 0, 10, 5100), (1500, 1200, 3, 5, 2000)])
def test_q6_matches_oracle(engine, params):

    t = dg.gen_fact(777_777, 18)
    li = dg.fact_to_storage_plan(t)
    assert engine.q6_lineitem_host(li, *params) == O.q6_lineitem(li, *params)


def test_q6_matches_reference_golden(engine):
    import json
    from pathlib import Path

    cases = json.loads((Path(__file__).parent / "golden" / "q6_reference.json").read_text())
    for c in cases:
        t = dg.gen_fact(c["n"], c["seed"])
        li = dg.fact_to_storage_plan(t)
        y, m, d = map(int, c["date"].split("-"))
        s = dg.days_from_civil(y, m, d) - 8035
        e = dg.days_from_civil(y + 1, m, d) - 8035
        disc = round(float(c["discount"]) * 100)
        q = round(float(c["quantity"]) * 100)
        rev, _ = engine.q6_lineitem_host(li, s, e, disc - 1, disc + 1, q)
        assert rev == c["revenue_raw"]
