"""Batched heterogeneous pipelines: many scan-agg / join / group-by instances in
one persistent kernel over a device work queue, captured in a CUDA graph
(``bo_batch_*`` in csrc/batch.cu), plus the tile-size autotuner and seeded
device-side generators for mixed workloads.

The reference runs one query per call (bespoke_tpch/query_impl.cpp:159-388);
batching has no reference counterpart, so every batched result is checked
against the solo run of the same instance (the solo runs are in turn checked
against the oracle by the pipeline tests).
"""
from __future__ import annotations

import ctypes as C
import json
import math
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import native as N
from .datagen import DATE_HI, DATE_LO

KINDS = {N.BATCH_SCAN_AGG: "scan_agg", N.BATCH_JOIN: "join", N.BATCH_GROUPBY: "groupby"}
TILE_CANDIDATES = (32768, 65536, 131072, 262144, 524288)
DEFAULT_TILE = 131072


# ------------------------------------------------------------ instances ----
@dataclass
class Instance:
    """One pipeline of a batch: its kind, device columns and constants."""
    kind: int
    rows: int                      # size class key (fact rows / probe rows / B rows)
    cols: dict                     # device tensors
    params: dict
    predicted: float = 0.0         # presizing prediction (<= 0: size for the upper bound)
    tile_rows: int = 0
    predicted_device: object = None  # device float tensor read at launch (overrides predicted)
    keep: list = field(default_factory=list)

    def to_c(self) -> N.BatchInstance:
        x = N.BatchInstance()
        x.kind = self.kind
        x.tile_rows = int(self.tile_rows)
        x.predicted = float(self.predicted)
        x.presize_factor = 0.0
        x.predicted_device = N.ptr(self.predicted_device) if self.predicted_device is not None else None
        p, c = self.params, self.cols
        if self.kind == N.BATCH_SCAN_AGG:
            x.fact = N.FactCols(*[N.ptr(c[k]) for k in ("ship_date", "quantity", "ext_price", "discount", "tax",
                                                         "flag_a", "flag_b")], int(c["ship_date"].numel()))
            x.ship_cutoff, x.n_flag_a, x.n_flag_b = p["cutoff"], p["n_flag_a"], p["n_flag_b"]
        elif self.kind == N.BATCH_JOIN:
            x.build = N.JoinBuildCols(N.ptr(c["b_key"]), N.ptr(c["b_date"]), N.ptr(c["b_seg"]),
                                      int(c["b_key"].numel()))
            x.probe = N.JoinProbeCols(N.ptr(c["p_fk"]), N.ptr(c["p_price"]), N.ptr(c["p_disc"]),
                                      int(c["p_fk"].numel()))
            x.join = N.JoinParams(p["date_lt"], p["seg_eq"])
        else:
            x.a = N.GbACols(N.ptr(c["a_ids"]), int(c["a_ids"].numel()))
            x.b = N.GbBCols(N.ptr(c["b_a"]), N.ptr(c["b_c"]), int(c["b_a"].numel()))
            x.c = N.GbCCols(N.ptr(c["c_cat"]), N.ptr(c["c_year"]), int(c["c_cat"].numel()))
            cats = list(p["cat_set"])
            for i, v in enumerate(cats):
                x.categories[i] = int(v)
            x.n_categories = len(cats)
            x.year_lo, x.year_hi, x.k, x.a_id_max = p["year_lo"], p["year_hi"], p["k"], p["a_id_max"]
        return x

    def algorithmic_bytes(self) -> int:
        c = self.cols
        return int(sum(t.numel() * t.element_size() for t in c.values()))


def result_dict(r: N.BatchResult, inst: Instance) -> dict:
    """The answer fields of one batched result (what must equal the solo run)."""
    if r.kind == N.BATCH_SCAN_AGG:
        ng = inst.params["n_flag_a"] * inst.params["n_flag_b"]
        return {"kind": "scan_agg", "groups": [r.q1[g].as_dict() for g in range(ng)], "reruns": r.reruns}
    if r.kind == N.BATCH_JOIN:
        d = r.join.as_dict()
        d["kind"] = "join"
        return d
    d = r.groupby.as_dict()
    d["kind"] = "groupby"
    return d


ANSWER_FIELDS = {
    "scan_agg": ("groups",),
    "join": ("build_rows", "distinct_keys", "match_count", "sum_exact", "sum_trunc"),
    "groupby": ("n_groups", "joined_rows", "c_qualifying", "keys", "counts", "min_years"),
}


def same_answer(a: dict, b: dict) -> bool:
    return all(a[f] == b[f] for f in ANSWER_FIELDS[a["kind"]])


# --------------------------------------------------------------- batch -----
def footprint(inst: Instance) -> tuple[int, int]:
    """(table bytes, work items) the instance needs in a batch."""
    tb, it = C.c_int64(), C.c_int64()
    x = inst.to_c()
    rc = N.lib().bo_batch_footprint(C.byref(x), C.byref(tb), C.byref(it))
    if rc != N.BO_OK:
        raise N.BoError(rc, "bo_batch_footprint")
    return int(tb.value), int(it.value)


class Batch:
    """A planned batch: tables allocated, work queue built, launch captured.

    ``Batch(engine, instances)`` sizes everything for those instances;
    ``Batch.pool(engine, max_instances, max_items, pool_bytes)`` makes an
    empty one that ``update`` re-plans in place (no re-capture)."""

    def __init__(self, engine, instances: list[Instance] | None, workers_per_sm: int = 0, _handle=None):
        self.engine = engine
        self._lib = N.lib()
        self.instances = list(instances or [])
        if _handle is not None:
            self.handle = _handle
            return
        arr = (N.BatchInstance * len(self.instances))(*[i.to_c() for i in self.instances])
        h = C.c_void_p()
        engine.ctx.call("bo_batch_create", arr, len(self.instances), int(workers_per_sm), C.byref(h))
        self.handle = h

    @classmethod
    def pool(cls, engine, max_instances: int, max_items: int, pool_bytes: int, workers_per_sm: int = 0) -> "Batch":
        h = C.c_void_p()
        engine.ctx.call("bo_batch_create_pool", int(max_instances), int(max_items), int(pool_bytes),
                        int(workers_per_sm), C.byref(h))
        return cls(engine, None, workers_per_sm, _handle=h)

    def update(self, instances: list[Instance]) -> None:
        arr = (N.BatchInstance * len(instances))(*[i.to_c() for i in instances])
        self.engine.ctx.call("bo_batch_update", self.handle, arr, len(instances))
        self.instances = list(instances)

    @property
    def num_items(self) -> int:
        return int(self._lib.bo_batch_num_items(self.handle))

    def launch(self) -> None:
        self.engine.ctx.call("bo_batch_launch", self.handle)

    def done(self) -> bool:
        """Non-blocking: has the last launch finished?"""
        rc = int(self._lib.bo_batch_done(self.handle))
        if rc < 0:
            raise N.BoError(rc, "bo_batch_done")
        return rc == 1

    def last_ms(self) -> float:
        return float(self._lib.bo_batch_last_ms(self.handle))

    def results(self) -> list[dict]:
        out = (N.BatchResult * len(self.instances))()
        self.engine.ctx.call("bo_batch_results", self.handle, out)
        return [result_dict(out[i], inst) for i, inst in enumerate(self.instances)]

    def run(self) -> list[dict]:
        self.launch()
        return self.results()

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.bo_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def solo_result(engine, inst: Instance, presized: bool = False) -> dict:
    """The same instance run alone through its standalone entry points (the
    plain exact-count form unless ``presized``)."""
    import torch

    c, p = inst.cols, inst.params
    if inst.kind == N.BATCH_SCAN_AGG:
        ng = p["n_flag_a"] * p["n_flag_b"]
        out = torch.zeros(ng * C.sizeof(N.Q1Agg), dtype=torch.uint8, device="cuda")
        cols = [c[k] for k in ("ship_date", "quantity", "ext_price", "discount", "tax", "flag_a", "flag_b")]
        engine.q1_fact_device(cols, int(c["ship_date"].numel()), p["cutoff"], p["n_flag_a"], p["n_flag_b"], out)
        engine.synchronize()
        host = out.cpu().numpy()
        aggs = (N.Q1Agg * ng).from_buffer_copy(host.tobytes())
        return {"kind": "scan_agg", "groups": [aggs[g].as_dict() for g in range(ng)], "reruns": 0}
    if inst.kind == N.BATCH_JOIN:
        build = (c["b_key"], c["b_date"], c["b_seg"])
        probe = (c["p_fk"], c["p_price"], c["p_disc"])
        nb, npr = int(c["b_key"].numel()), int(c["p_fk"].numel())
        if presized:
            pred = torch.tensor([inst.predicted], dtype=torch.float32, device="cuda")
            d = engine.join_presized(build, probe, nb, npr, p["date_lt"], p["seg_eq"], pred)
        else:
            d = engine.join_plain(build, probe, nb, npr, p["date_lt"], p["seg_eq"])
        d["kind"] = "join"
        return d
    a, b, cc, prm, keep = engine.gb_args(c["a_ids"], c["b_a"], c["b_c"], c["c_cat"], c["c_year"],
                                         int(c["a_ids"].numel()), int(c["b_a"].numel()), int(c["c_cat"].numel()),
                                         p["cat_set"], p["year_lo"], p["year_hi"], p["k"], p["a_id_max"])
    out = N.GbResult()
    if presized:
        pred = torch.tensor([inst.predicted], dtype=torch.float32, device="cuda")
        engine.ctx.call("bo_groupby_topk_presized", C.byref(a), C.byref(b), C.byref(cc), C.byref(prm),
                        C.c_void_p(pred.data_ptr()), C.byref(out))
    else:
        engine.ctx.call("bo_groupby_topk_plain", C.byref(a), C.byref(b), C.byref(cc), C.byref(prm), C.byref(out))
    d = out.as_dict()
    d["kind"] = "groupby"
    return d


# ----------------------------------------------------------- generators ----
def _gen(seed: int):
    import torch

    g = torch.Generator(device="cuda")
    g.manual_seed(int(seed))
    return g


def _randint(g, lo: int, hi: int, n: int, dtype):
    """Uniform integers in [lo, hi] (inclusive) on the device."""
    import torch

    return torch.randint(lo, hi + 1, (n,), generator=g, device="cuda", dtype=torch.int64).to(dtype)


def fact_instance(n: int, seed: int, cutoff: int | None = None) -> Instance:
    """Scan-filter-group-aggregate instance: the fact-table distributions of the
    6M-row workload (ship_date uniform over the TPC-H range, quantity 1..50,
    price 900.00..105000.00, discount 0..10, tax 0..8, flag_a 0..2, flag_b 0..1)
    scaled to n rows; the cutoff is redrawn per instance unless given."""
    import torch

    g = _gen(seed)
    rng = np.random.default_rng(seed)
    cols = {
        "ship_date": _randint(g, DATE_LO, DATE_HI, n, torch.int32),
        "quantity": _randint(g, 1, 50, n, torch.int64) * 100,
        "ext_price": _randint(g, 90_000, 10_500_000, n, torch.int64),
        "discount": _randint(g, 0, 10, n, torch.int64),
        "tax": _randint(g, 0, 8, n, torch.int64),
        "flag_a": _randint(g, 0, 2, n, torch.uint8),
        "flag_b": _randint(g, 0, 1, n, torch.uint8),
    }
    cut = int(rng.integers(DATE_LO + 365, DATE_HI)) if cutoff is None else cutoff
    return Instance(N.BATCH_SCAN_AGG, n, cols, {"cutoff": cut, "n_flag_a": 3, "n_flag_b": 2})


def join_instance(n_probe: int, seed: int, n_build: int | None = None, date_lt: int | None = None,
                  seg_eq: int | None = None) -> Instance:
    """Filtered join instance: unique shuffled build keys (n_build = n_probe / 4
    unless given), uniform build dates and segments 0..4, probe keys uniform
    over the build keys; date cutoff and segment redrawn per instance."""
    import torch

    nb = max(1, n_probe // 4) if n_build is None else n_build
    g = _gen(seed)
    rng = np.random.default_rng(seed + 7919)
    cols = {
        "b_key": (torch.randperm(nb, generator=g, device="cuda") + 1).to(torch.int32),
        "b_date": _randint(g, DATE_LO, DATE_HI, nb, torch.int32),
        "b_seg": _randint(g, 0, 4, nb, torch.uint8),
        "p_fk": _randint(g, 1, max(nb, 1), n_probe, torch.int32),
        "p_price": _randint(g, 90_000, 10_500_000, n_probe, torch.int64),
        "p_disc": _randint(g, 0, 10, n_probe, torch.int64),
    }
    dl = int(rng.integers(DATE_LO + 100, DATE_HI)) if date_lt is None else date_lt
    se = int(rng.integers(0, 5)) if seg_eq is None else seg_eq
    return Instance(N.BATCH_JOIN, n_probe, cols, {"date_lt": dl, "seg_eq": se})


def _zipf_device(g, n: int, n_ranks: int, s: float):
    """n draws of a bounded Zipf law over ranks 0..n_ranks-1 by inverse CDF."""
    import torch

    w = torch.arange(1, n_ranks + 1, dtype=torch.float64, device="cuda").pow(-s)
    cdf = torch.cumsum(w, 0)
    cdf /= cdf[-1].clone()
    u = torch.rand(n, generator=g, device="cuda", dtype=torch.float64)
    return torch.clamp(torch.searchsorted(cdf, u, right=True), max=n_ranks - 1)


def groupby_tables_device(n_a: int, n_b: int, n_c: int, seed: int, s_a: float = 1.1, s_c: float = 0.9) -> dict:
    """Device tables of the skewed three-way join: A ids 1..n_a shuffled, B
    (a_id Zipf s_a over A, c_id Zipf s_c over C rows; ranks mapped to ids by
    seeded permutations), C (category 0..112, year 1900..2020)."""
    import torch

    g = _gen(seed)
    a_ids = (torch.randperm(n_a, generator=g, device="cuda") + 1).to(torch.int32)
    rank_to_a = (torch.randperm(n_a, generator=g, device="cuda") + 1).to(torch.int32)
    rank_to_c = torch.randperm(n_c, generator=g, device="cuda").to(torch.int32)
    return {
        "a_ids": a_ids,
        "b_a": rank_to_a[_zipf_device(g, n_b, n_a, s_a)].contiguous(),
        "b_c": rank_to_c[_zipf_device(g, n_b, n_c, s_c)].contiguous(),
        "c_cat": _randint(g, 0, 112, n_c, torch.int16),  # uint16 values 0..112, same bits
        "c_year": _randint(g, 1900, 2020, n_c, torch.int32),
        "a_id_max": n_a,
    }


def groupby_instance(n_b: int, seed: int, k: int = 10) -> Instance:
    """Skewed three-way join + group-by + top-k instance: A, B, C in the
    2.5M : 36M : 4M proportions of the full workload scaled to n_b B rows,
    a_id Zipf s=1.1 over A, c_id Zipf s=0.9 over C, category 0..112, year
    1900..2020; the category set (8 values) and the year range are redrawn."""
    n_a = max(16, int(round(n_b * 2.5 / 36)))
    n_c = max(16, int(round(n_b * 4 / 36)))
    rng = np.random.default_rng(seed + 104729)
    cols = groupby_tables_device(n_a, n_b, n_c, seed)
    del cols["a_id_max"]
    cat_set = sorted(int(v) for v in rng.choice(113, size=8, replace=False))
    y0 = int(rng.integers(1900, 2010))
    y1 = int(min(2020, y0 + int(rng.integers(5, 30))))
    params = {"cat_set": cat_set, "year_lo": y0, "year_hi": y1, "k": k, "a_id_max": n_a}
    return Instance(N.BATCH_GROUPBY, n_b, cols, params)


def mixed_workload(n_instances: int = 64, lo: float = 1e4, hi: float = 6e7, seed: int = 0,
                   kinds=(N.BATCH_SCAN_AGG, N.BATCH_JOIN, N.BATCH_GROUPBY)) -> list[Instance]:
    """Instances drawn from the three pipeline shapes with row counts
    log-uniform in [lo, hi] (seeded) and predicate constants redrawn."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_instances):
        kind = int(kinds[int(rng.integers(0, len(kinds)))])
        rows = int(math.exp(rng.uniform(math.log(lo), math.log(hi))))
        s = int(rng.integers(0, 2**31 - 1))
        if kind == N.BATCH_SCAN_AGG:
            out.append(fact_instance(rows, s))
        elif kind == N.BATCH_JOIN:
            out.append(join_instance(rows, s))
        else:
            out.append(groupby_instance(rows, s))
    return out


# ------------------------------------------------------------ autotuner ----
def size_bucket(rows: int) -> int:
    """Size class of an instance: floor(log10(rows)), clamped to [4, 8]."""
    return int(min(8, max(4, math.floor(math.log10(max(rows, 1))))))


@dataclass
class TileTable:
    """Autotuned tile sizes: tiles[kind][bucket] -> rows per work item, and
    the worker blocks per SM of the persistent kernel."""
    tiles: dict = field(default_factory=dict)
    workers_per_sm: int = 0
    measured: dict = field(default_factory=dict)

    def tile_for(self, kind: int, rows: int) -> int:
        return int(self.tiles.get(str(kind), {}).get(str(size_bucket(rows)), DEFAULT_TILE))

    def apply(self, instances: list[Instance]) -> None:
        for inst in instances:
            inst.tile_rows = self.tile_for(inst.kind, inst.rows)

    def to_json(self) -> str:
        return json.dumps({"tiles": self.tiles, "workers_per_sm": self.workers_per_sm, "measured": self.measured},
                          sort_keys=True)

    @classmethod
    def from_json(cls, s: str) -> "TileTable":
        d = json.loads(s)
        return cls(d.get("tiles", {}), int(d.get("workers_per_sm", 0)), d.get("measured", {}))

    def save(self, path: Path) -> None:
        Path(path).write_text(self.to_json())

    @classmethod
    def load(cls, path: Path) -> "TileTable":
        return cls.from_json(Path(path).read_text())


def time_batch(engine, instances: list[Instance], workers_per_sm: int = 0, reps: int = 3) -> float:
    """Median device time (ms) of one graph launch of the batch."""
    b = Batch(engine, instances, workers_per_sm)
    try:
        b.launch()
        b.results()
        ts = []
        for _ in range(reps):
            b.launch()
            engine.synchronize()
            ts.append(b.last_ms())
        return float(np.median(ts))
    finally:
        b.close()


def autotune(engine, instances: list[Instance], candidates=TILE_CANDIDATES, workers=(1, 2), reps: int = 3,
             timer=time_batch) -> TileTable:
    """Picks, for every (kind, size bucket) present, the tile size whose batch
    of just those instances runs fastest, then the worker count for the whole
    mix with the chosen tiles.  ``timer(engine, instances, workers_per_sm,
    reps)`` returns milliseconds (injectable for tests)."""
    table = TileTable()
    groups: dict[tuple[int, int], list[Instance]] = {}
    for inst in instances:
        groups.setdefault((inst.kind, size_bucket(inst.rows)), []).append(inst)
    for (kind, bucket), insts in sorted(groups.items()):
        best, best_ms = None, math.inf
        for t in candidates:
            for inst in insts:
                inst.tile_rows = t
            ms = timer(engine, insts, 0, reps)
            table.measured[f"{KINDS[kind]}/1e{bucket}/{t}"] = ms
            if ms < best_ms:
                best, best_ms = t, ms
        table.tiles.setdefault(str(kind), {})[str(bucket)] = int(best)
    table.apply(instances)
    best_w, best_ms = 0, math.inf
    for w in workers:
        ms = timer(engine, instances, w, reps)
        table.measured[f"workers/{w}"] = ms
        if ms < best_ms:
            best_w, best_ms = w, ms
    table.workers_per_sm = best_w
    return table


# ------------------------------------------------------------------ CLI ----
TILE_TABLE_PATH = Path(__file__).resolve().parent / "tile_table.json"


def load_tile_table() -> TileTable:
    """The autotuned table shipped with the package (defaults if absent)."""
    return TileTable.load(TILE_TABLE_PATH) if TILE_TABLE_PATH.exists() else TileTable()


def main(argv=None) -> None:
    """``python -m bespokeolap_artifacts_b200.batching --autotune OUT.json``:
    tunes the tile table on the 64-instance mixed workload (seeded) on cuda:0."""
    import argparse

    import torch

    from .engine import Engine

    ap = argparse.ArgumentParser()
    ap.add_argument("--autotune", required=True, help="output JSON path")
    ap.add_argument("--instances", type=int, default=64)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--reps", type=int, default=3)
    a = ap.parse_args(argv)
    torch.cuda.set_device(0)
    eng = Engine(0)
    insts = mixed_workload(a.instances, seed=a.seed)
    table = autotune(eng, insts, reps=a.reps)
    table.save(Path(a.autotune))
    print(table.to_json())
    eng.close()


if __name__ == "__main__":
    main()
