"""Batched heterogeneous pipelines (one persistent kernel over a device work
queue, CUDA graph): every instance's answer must equal its solo run exactly,
for empty and ragged tables, many tiles per stage, under-predicted tables
(overflow -> exact rerun) and repeated launches of the same graph."""
import pytest

from bespokeolap_artifacts_b200 import batching as B
from bespokeolap_artifacts_b200 import native as N

pytestmark = pytest.mark.gpu


def mixed_small():
    insts = [
        B.fact_instance(0, 1),
        B.fact_instance(3, 2),
        B.fact_instance(10_001, 3),
        B.fact_instance(300_007, 4),
        B.join_instance(0, 5, n_build=100),
        B.join_instance(5_000, 6),
        B.join_instance(200_001, 7, n_build=50_003),
        B.join_instance(150_000, 8),
        B.groupby_instance(20_000, 9),
        B.groupby_instance(400_003, 10),
        B.groupby_instance(90_000, 11, k=64),
        B.groupby_instance(50_000, 12, k=0),
    ]
    return insts


def check_against_solo(engine, insts, results):
    for i, (inst, r) in enumerate(zip(insts, results)):
        s = B.solo_result(engine, inst)
        assert B.same_answer(r, s), (i, B.KINDS[inst.kind], r, s)


def test_batch_matches_solo_upper_bound_tables(engine, torch_cuda):
    insts = mixed_small()
    b = B.Batch(engine, insts)
    assert b.num_items >= len(insts)
    res = b.run()
    check_against_solo(engine, insts, res)
    assert all(r["reruns"] == 0 for r in res)
    b.close()


def test_batch_small_tiles_many_items(engine, torch_cuda):
    insts = mixed_small()
    for inst in insts:
        inst.tile_rows = 4096
    b = B.Batch(engine, insts, workers_per_sm=1)
    res = b.run()
    check_against_solo(engine, insts, res)
    # The same graph launched again starts from a clean state.
    res2 = b.run()
    assert all(B.same_answer(x, y) for x, y in zip(res, res2))
    b.close()


def test_batch_presized_and_overflow_rerun(engine, torch_cuda):
    wide = {"year_lo": 1900, "year_hi": 2020}  # enough groups to overflow the minimum table
    j = B.join_instance(120_000, 21)
    g = B.groupby_instance(300_000, 22)
    g.params.update(wide)
    exact_j = B.solo_result(engine, j)
    exact_g = B.solo_result(engine, g)
    assert exact_j["distinct_keys"] > 1024 * 7 // 8 and exact_g["n_groups"] > 1024 * 7 // 8
    # Accurate predictions: presized tables, no rerun.
    j.predicted = float(exact_j["build_rows"])
    g.predicted = float(exact_g["n_groups"])
    # Far too low: the table overflows and the instance is rerun exactly.
    j_low = B.join_instance(120_000, 21)
    j_low.predicted = 1.0
    g_low = B.groupby_instance(300_000, 22)
    g_low.params.update(wide)
    g_low.predicted = 1.0
    insts = [j, g, j_low, g_low, B.fact_instance(70_000, 23)]
    res = B.Batch(engine, insts).run()
    check_against_solo(engine, insts, res)
    assert res[0]["reruns"] == 0 and res[1]["reruns"] == 0
    assert res[2]["reruns"] == 1 and res[3]["reruns"] == 1
    # The batched presized forms equal the solo presized forms too.
    assert B.same_answer(res[0], B.solo_result(engine, j, presized=True))
    assert B.same_answer(res[1], B.solo_result(engine, g, presized=True))


def test_batch_log_uniform_mix(engine, torch_cuda):
    insts = B.mixed_workload(24, lo=1e4, hi=2e6, seed=5)
    res = B.Batch(engine, insts).run()
    check_against_solo(engine, insts, res)


def test_batch_rejects_bad_instances(engine, torch_cuda):
    inst = B.fact_instance(1000, 1)
    inst.params["n_flag_a"] = 5  # 5 x 2 groups > 8
    with pytest.raises(N.BoError):
        B.Batch(engine, [inst])
    g = B.groupby_instance(1000, 2)
    g.params["k"] = 65
    with pytest.raises(N.BoError):
        B.Batch(engine, [g])


def test_autotuner_picks_measured_best(engine, torch_cuda):
    insts = B.mixed_workload(6, lo=1e5, hi=1e6, seed=9)
    table = B.autotune(engine, insts, candidates=(32768, 131072), workers=(1, 2), reps=1)
    for (key, ms) in table.measured.items():
        assert ms > 0, key
    res = B.Batch(engine, insts, table.workers_per_sm).run()
    check_against_solo(engine, insts, res)


def test_batch_pool_replans_in_place(engine, torch_cuda):
    sets = [B.mixed_workload(8, lo=1e4, hi=5e5, seed=s) for s in (31, 32, 33)]
    need_bytes = max(sum(B.footprint(i)[0] for i in insts) for insts in sets)
    need_items = max(sum(B.footprint(i)[1] for i in insts) for insts in sets)
    b = B.Batch.pool(engine, 8, need_items, need_bytes)
    for insts in sets + sets[:1]:
        b.update(insts)
        res = b.run()
        check_against_solo(engine, insts, res)
    # Too many tables for the pool: refused, the batch stays usable.
    big = B.mixed_workload(8, lo=2e6, hi=4e6, seed=34, kinds=(N.BATCH_JOIN,))
    if sum(B.footprint(i)[0] for i in big) > need_bytes:
        with pytest.raises(N.BoError):
            b.update(big)
    b.update(sets[1])
    check_against_solo(engine, sets[1], b.run())
    b.close()


def test_batch_device_prediction(engine, torch_cuda):
    """Capacity taken from a device float at launch time (an MLP output left on
    the device): same capacity as the solo presized form, same answer; the
    same graph re-run with a too-low value overflows and is rerun exactly."""
    torch = torch_cuda
    g = B.groupby_instance(300_000, 41)
    g.params.update({"year_lo": 1900, "year_hi": 2020})
    j = B.join_instance(200_000, 42)
    exact_g, exact_j = B.solo_result(engine, g), B.solo_result(engine, j)
    pred = torch.tensor([float(exact_g["n_groups"]), float(exact_j["build_rows"])], dtype=torch.float32,
                        device="cuda")
    g.predicted_device, j.predicted_device = pred[0:1], pred[1:2]
    g.predicted, j.predicted = float(exact_g["n_groups"]), float(exact_j["build_rows"])
    torch.cuda.synchronize()  # the engine's stream reads what torch's stream wrote
    b = B.Batch(engine, [g, j])
    res = b.run()
    check_against_solo(engine, [g, j], res)
    solo_g, solo_j = B.solo_result(engine, g, presized=True), B.solo_result(engine, j, presized=True)
    assert res[0]["capacity_log2"] == solo_g["capacity_log2"] and res[0]["reruns"] == 0
    assert res[1]["capacity_log2"] == solo_j["capacity_log2"] and res[1]["reruns"] == 0
    pred.fill_(1.0)
    torch.cuda.synchronize()
    res = b.run()
    check_against_solo(engine, [g, j], res)
    assert res[0]["reruns"] == 1 and res[1]["reruns"] == 1
    b.close()
