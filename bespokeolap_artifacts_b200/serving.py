"""Serving loop over device-resident tables with continuous batching.

Requests (scan-agg, join or group-by queries with their own predicate
constants) arrive as a Poisson stream.  The server keeps a FIFO of arrived
requests and several batch slots -- each its own engine context (CUDA stream)
and a re-plannable persistent-kernel batch with a fixed table pool.  Whenever a
slot is free and requests are waiting, it admits requests in arrival order
while their tables, sized from the MLP predictions (the calibrated sizers),
fit the slot's HBM pool and work-item budget, re-plans the batch in place and
launches it; slots run concurrently on the device, so requests that arrive
while others are on the GPU start as soon as a slot and memory free up.  A
finished slot's results are read (an instance whose presized table overflowed
is rerun exactly) and the slot takes the next requests.

The baseline runs the same arrival stream one pipeline per launch: each
request alone, in arrival order, through the plain exact-count entry points.

The reference serves one query per call (bespoke_tpch/query_impl.cpp:159-388);
this layer has no reference counterpart.  Every served answer must equal the
request's solo answer (tests/test_serving_gpu.py).
"""
from __future__ import annotations

import ctypes as C
import math
import time
from collections import deque
from dataclasses import dataclass, field
from types import SimpleNamespace

import numpy as np

from . import batching as B
from . import native as N
from .datagen import DATE_HI, DATE_LO

KIND_NAMES = B.KINDS


# ----------------------------------------------------------------- tables ---
@dataclass
class ServingTables:
    """The device-resident tables every request reads, plus their load-time
    statistics (sketches) for the sizers."""
    fact: dict
    join: dict
    gb: dict
    join_stats: object = None
    gb_stats: object = None

    @classmethod
    def load(cls, engine, fact_rows: int = 60_000_000, seed: int = 0) -> "ServingTables":
        """fact_rows fact rows (scan-agg distributions); a join with a build
        side of fact_rows / 4 rows (ten times the 1.5M build of the join
        workload at 60M) and a probe side of fact_rows rows; a group-by with B
        = fact_rows rows and A, C ten times the 2.5M / 4M of the group-by
        workload at 60M (scaled down proportionally for smaller fact_rows)."""
        import torch

        from . import learned as L

        f = B.fact_instance(fact_rows, seed + 1).cols
        j = B.join_instance(fact_rows, seed + 2, n_build=max(1, fact_rows // 4)).cols
        scale = fact_rows / 60_000_000
        n_a, n_c = max(16, int(25_000_000 * scale)), max(16, int(40_000_000 * scale))
        g = B.groupby_tables_device(n_a, fact_rows, n_c, seed + 3)
        # A's id mask depends on table A alone: built once at load (an index,
        # like the sketches) for the slots' group-by pipelines.
        g["a_mask"] = torch.zeros((int(g["a_id_max"]) + 32) // 32, dtype=torch.int32, device="cuda")
        engine.ctx.call("bo_groupby_a_mask_device", C.byref(N.GbACols(N.ptr(g["a_ids"]), int(g["a_ids"].numel()))),
                        int(g["a_id_max"]), C.c_void_p(g["a_mask"].data_ptr()))
        t = cls(f, j, g)
        t.join_stats = L.join_table_stats(engine.ctx, j["b_key"], j["b_date"], j["b_seg"], int(j["b_key"].numel()))
        t.gb_stats = L.groupby_table_stats(engine.ctx, g, n_a, fact_rows, n_c)
        return t


# --------------------------------------------------------------- requests ---
@dataclass
class Request:
    rid: int
    kind: int
    params: dict
    arrival: float                      # seconds from the start of the stream
    predicted: float = 0.0              # sizing prediction (join rows / groups)
    result: dict | None = None
    done: float = math.nan              # completion time, same clock as arrival

    @property
    def latency_ms(self) -> float:
        return (self.done - self.arrival) * 1e3


def poisson_requests(rate_qps: float, n: int, seed: int = 0, mix=(1, 1, 1)) -> list[Request]:
    """n requests with exponential inter-arrival times at rate_qps, the three
    pipeline shapes drawn with weights `mix`, predicate constants seeded."""
    rng = np.random.default_rng(seed)
    kinds = (N.BATCH_SCAN_AGG, N.BATCH_JOIN, N.BATCH_GROUPBY)
    w = np.asarray(mix, np.float64) / float(sum(mix))
    t = 0.0
    out = []
    for i in range(n):
        t += float(rng.exponential(1.0 / rate_qps))
        kind = int(kinds[int(rng.choice(3, p=w))])
        if kind == N.BATCH_SCAN_AGG:
            p = {"cutoff": int(rng.integers(DATE_LO + 365, DATE_HI + 1)), "n_flag_a": 3, "n_flag_b": 2}
        elif kind == N.BATCH_JOIN:
            p = {"date_lt": int(rng.integers(DATE_LO + 100, DATE_HI + 1)), "seg_eq": int(rng.integers(0, 5))}
        else:
            y0 = int(rng.integers(1900, 2010))
            p = {"cat_set": sorted(int(v) for v in rng.choice(113, size=8, replace=False)), "year_lo": y0,
                 "year_hi": int(min(2020, y0 + int(rng.integers(5, 30)))), "k": 10}
        out.append(Request(i, kind, p, t))
    return out


def instance_of(tables: ServingTables, r: Request, tile_table: B.TileTable | None = None) -> B.Instance:
    """The batch instance of a request over the shared device tables."""
    if r.kind == N.BATCH_SCAN_AGG:
        cols, rows = tables.fact, int(tables.fact["ship_date"].numel())
        params = dict(r.params)
    elif r.kind == N.BATCH_JOIN:
        cols, rows = tables.join, int(tables.join["p_fk"].numel())
        params = dict(r.params)
    else:
        cols = {k: v for k, v in tables.gb.items() if k not in ("a_id_max", "a_mask")}
        rows = int(cols["b_a"].numel())
        params = dict(r.params, a_id_max=int(tables.gb["a_id_max"]))
    inst = B.Instance(r.kind, rows, cols, params, predicted=r.predicted)
    if tile_table is not None:
        inst.tile_rows = tile_table.tile_for(r.kind, rows)
    return inst


def predict_requests(tables: ServingTables, reqs: list[Request], join_sizer=None, gb_sizer=None) -> None:
    """Fills r.predicted from the sizers (one device inference per kind)."""
    from . import learned as L

    js = [r for r in reqs if r.kind == N.BATCH_JOIN]
    gs = [r for r in reqs if r.kind == N.BATCH_GROUPBY]
    if js and join_sizer is not None:
        x = np.stack([L.join_features(tables.join_stats, r.params["date_lt"], r.params["seg_eq"]) for r in js])
        for r, p in zip(js, join_sizer.predict_host(x)):
            r.predicted = float(p)
    if gs and gb_sizer is not None:
        x = np.stack([L.groupby_features(tables.gb_stats, r.params["cat_set"], r.params["year_lo"],
                                         r.params["year_hi"]) for r in gs])
        for r, p in zip(gs, gb_sizer.predict_host(x)[:, 0]):
            r.predicted = float(p)


def admit(pending: deque, footprints: dict, max_batch: int, pool_bytes: int, max_items: int,
          kind: int | None = None) -> list:
    """Takes requests from the head of `pending` (arrival order) while the
    batch stays within max_batch requests, pool_bytes of tables and max_items
    work items.  footprints[rid] = (table bytes, items).  A request whose
    footprint alone exceeds the slot is admitted alone (its tables are then
    sized for the upper bound by the caller) so nothing starves.  With `kind`
    set, only requests of that kind are taken (in arrival order); the others
    keep their places."""
    out, tb, it = [], 0, 0
    if kind is None:
        while pending and len(out) < max_batch:
            r = pending[0]
            b, i = footprints[r.rid]
            if out and (tb + b > pool_bytes or it + i > max_items):
                break
            out.append(pending.popleft())
            tb += b
            it += i
        return out
    keep = deque()
    while pending:
        r = pending.popleft()
        b, i = footprints[r.rid]
        if r.kind != kind or len(out) >= max_batch or (out and (tb + b > pool_bytes or it + i > max_items)):
            keep.append(r)
            continue
        out.append(r)
        tb += b
        it += i
    pending.extend(keep)
    return out


# Service order of the kinds under the short-first policy: scan-agg (a single
# streaming pass, ~0.4 ms on the serving tables) before the join and the
# group-by (~1 ms each).
SHORT_FIRST = (N.BATCH_SCAN_AGG, N.BATCH_JOIN, N.BATCH_GROUPBY)


def next_kind(pending: deque, policy: str, waited_ms: float, max_wait_ms: float) -> int | None:
    """The kind a free slot takes next: None (arrival order, mixed kinds) for
    "fifo"; for "short_first" the shortest kind waiting, unless the oldest
    request has waited longer than max_wait_ms (then its kind: no starvation)."""
    if policy != "short_first" or not pending:
        return None
    if waited_ms > max_wait_ms:
        return pending[0].kind
    present = {r.kind for r in pending}
    for k in SHORT_FIRST:
        if k in present:
            return k
    return pending[0].kind


# ----------------------------------------------------------------- server ---
@dataclass
class Slot:
    engine: object
    batch: B.Batch
    stream: object = None               # torch stream the slot's engine runs on
    join_out: object = None             # device records of the slot's shared joins
    gb_out: object = None               # device records of the slot's group-by pipelines
    gb_pred_h: object = None            # their predicted group counts (pinned host, device)
    gb_pred_d: object = None
    event: object = None                # recorded after the slot's last launch
    q1_out: object = None               # device groups of a lone scan-agg request
    pred_h: object = None               # pinned / device table size of a lone join request
    pred_d: object = None
    cnt_d: object = None                # a lone join's exact qualifying-row count (device)
    reqs: list = field(default_factory=list)
    joins: list = field(default_factory=list)
    gbs: list = field(default_factory=list)
    others: list = field(default_factory=list)
    lone: object = None                 # a request run alone through its standalone kernels
    busy: bool = False


class BatchedServer:
    """Continuous batching over `n_slots` concurrently running batch slots.

    The join requests a slot admits share one pass over the join tables
    (bo_join_multi_device: one build and one probe pass whatever their number,
    since they differ only in predicate constants); each group-by request runs
    the presized multi-kernel pipeline (table sized on the device from its MLP
    prediction, A's id mask built once at load; an overflowed table is rerun
    exactly), and the scan-agg requests run as instances of the slot's
    persistent batch kernel -- all on the slot's stream, one event at the
    end.  A request that finds an idle slot with nothing else waiting runs
    alone through its standalone kernel (scan-agg) or the join sized from its
    exact count on the device (count kernel, then the presized pipeline).
    With shared=False every request is a batch instance.

    Admission policy: "fifo" takes waiting requests in arrival order, kinds
    mixed; "short_first" fills a free slot with requests of one kind only,
    the shortest kind waiting first (scan-agg, join, group-by), unless the
    oldest request has waited max_wait_ms, so that a short request neither
    waits behind nor completes with a long one in the same slot.  Spill: with
    a slot running, an idle one starts only once spill_queue requests wait or
    the oldest has waited spill_wait_ms."""

    def __init__(self, tables: ServingTables, n_slots: int = 2, max_batch: int = 16,
                 pool_bytes: int = 2 << 30, max_items: int = 65536, workers_per_sm: int = 1,
                 join_sizer=None, gb_sizer=None, tile_table: B.TileTable | None = None, shared: bool = True,
                 policy: str = "fifo", max_wait_ms: float = 4.0, spill_queue: int = 1,
                 spill_wait_ms: float = 1.0, batch_from: int = 1):
        import torch

        from .engine import Engine

        self.tables = tables
        self.max_batch, self.pool_bytes, self.max_items = max_batch, pool_bytes, max_items
        self.join_sizer, self.gb_sizer = join_sizer, gb_sizer
        self.tile_table = tile_table
        self.shared = shared
        if policy not in ("fifo", "short_first"):
            raise ValueError(f"unknown admission policy {policy!r}")
        self.policy, self.max_wait_ms = policy, max_wait_ms
        # While a slot is running, another one starts only once spill_queue
        # requests wait or the oldest has waited spill_wait_ms: at low load a
        # request then waits a little for the running one instead of sharing
        # the GPU with it (two pipelines that each stream 1-2 GB slow each
        # other down by more than the wait).  spill_queue=1: start at once.
        self.spill_queue, self.spill_wait_ms = max(1, int(spill_queue)), spill_wait_ms
        # While fewer than batch_from requests wait, a free slot takes one (run
        # alone, as one pipeline per launch would): a batch of two or three
        # makes its first request wait for all of them, which only pays once
        # the queue is long.  batch_from=1: always batch what is waiting.
        self.batch_from = max(1, int(batch_from))
        self.slots = []
        for _ in range(n_slots):
            e = Engine(0)
            st = torch.cuda.Stream()
            e.set_stream(st.cuda_stream)
            out = torch.zeros(N.JOIN_MULTI_MAX * C.sizeof(N.JoinResult), dtype=torch.uint8, device="cuda")
            slot = Slot(e, B.Batch.pool(e, max_batch, max_items, pool_bytes, workers_per_sm), st, out)
            slot.gb_out = torch.zeros(max_batch * C.sizeof(N.GbResult), dtype=torch.uint8, device="cuda")
            slot.gb_pred_h = torch.zeros(max_batch, dtype=torch.float32).pin_memory()
            slot.gb_pred_d = torch.zeros(max_batch, dtype=torch.float32, device="cuda")
            slot.q1_out = torch.zeros(N.Q1_MAX_GROUPS * C.sizeof(N.Q1Agg), dtype=torch.uint8, device="cuda")
            slot.pred_h = torch.zeros(1, dtype=torch.float32).pin_memory()
            slot.pred_d = torch.zeros(1, dtype=torch.float32, device="cuda")
            slot.cnt_d = torch.zeros(1, dtype=torch.int64, device="cuda")
            self.slots.append(slot)
        self.launches = 0

    def close(self):
        for s in self.slots:
            s.batch.close()
            s.engine.close()

    def _footprint(self, r: Request) -> tuple[int, int]:
        if self.shared and r.kind == N.BATCH_JOIN:
            return 0, 0  # shared joins use the slot's own table, not the batch pool
        tb, items = B.footprint(instance_of(self.tables, r, self.tile_table))
        if self.shared and r.kind == N.BATCH_GROUPBY:
            return tb, 0  # its own pipeline: HBM footprint from the prediction, no batch work items
        return tb, items

    def _launch_lone(self, s: Slot, r: Request) -> None:
        """A request that finds an idle slot and no other request waiting runs
        alone through its standalone kernels (the scan-agg kernel; the count
        kernel, then the join sized from it on the device), not through the batch machinery: at low load nothing
        is there to share, and the batch kernel's re-plan would only add to
        its latency."""
        import torch

        s.lone = r
        if r.kind == N.BATCH_SCAN_AGG:
            f, p = self.tables.fact, r.params
            cols = [f[k] for k in ("ship_date", "quantity", "ext_price", "discount", "tax", "flag_a", "flag_b")]
            s.engine.q1_fact_device(cols, int(f["ship_date"].numel()), p["cutoff"], p["n_flag_a"], p["n_flag_b"],
                                    s.q1_out)
        else:
            # A lone join sized from its exact count without a host round trip:
            # the count kernel, the count turned into the presized path's size
            # input on the device, then the presized pipeline (4 slots per
            # qualifying row: the plain form's table), all enqueued at once.
            j = self.tables.join
            s.engine.join_count_device((j["b_key"], j["b_date"], j["b_seg"]), int(j["b_key"].numel()),
                                       r.params["date_lt"], r.params["seg_eq"], s.cnt_d)
            with torch.cuda.stream(s.stream):
                s.pred_d.copy_(s.cnt_d.to(torch.float32).clamp_(min=1.0))
            s.engine.join_presized_device((j["b_key"], j["b_date"], j["b_seg"]),
                                          (j["p_fk"], j["p_price"], j["p_disc"]), int(j["b_key"].numel()),
                                          int(j["p_fk"].numel()), r.params["date_lt"], r.params["seg_eq"], s.pred_d,
                                          s.join_out)

    def _launch(self, s: Slot, reqs: list) -> None:
        """Enqueues one slot's requests on its stream: the shared joins, then
        the batch kernel over the rest; an event marks the end."""
        import torch

        s.lone = None
        if self.shared and len(reqs) == 1 and reqs[0].kind in (N.BATCH_SCAN_AGG, N.BATCH_JOIN):
            s.joins, s.gbs, s.others = [], [], []
            self._launch_lone(s, reqs[0])
            s.event = torch.cuda.Event()
            s.event.record(s.stream)
            s.reqs, s.busy = reqs, True
            self.launches += 1
            return
        s.joins = [r for r in reqs if self.shared and r.kind == N.BATCH_JOIN]
        s.gbs = [r for r in reqs if self.shared and r.kind == N.BATCH_GROUPBY]
        s.others = [r for r in reqs if not (self.shared and r.kind in (N.BATCH_JOIN, N.BATCH_GROUPBY))]
        if s.gbs:
            for i, r in enumerate(s.gbs):
                s.gb_pred_h[i] = float(r.predicted)
            with torch.cuda.stream(s.stream):
                s.gb_pred_d[: len(s.gbs)].copy_(s.gb_pred_h[: len(s.gbs)], non_blocking=True)
            g = self.tables.gb
            for i, r in enumerate(s.gbs):
                prm = SimpleNamespace(cat_set=r.params["cat_set"], year_lo=r.params["year_lo"],
                                      year_hi=r.params["year_hi"], k=r.params["k"])
                s.engine.groupby_presized_device(g, prm, s.gb_pred_d[i:i + 1],
                                                 s.gb_out[i * C.sizeof(N.GbResult):(i + 1) * C.sizeof(N.GbResult)])
        if s.joins:
            j = self.tables.join
            s.engine.join_multi_device((j["b_key"], j["b_date"], j["b_seg"]), (j["p_fk"], j["p_price"], j["p_disc"]),
                                       int(j["b_key"].numel()), int(j["p_fk"].numel()),
                                       [(r.params["date_lt"], r.params["seg_eq"]) for r in s.joins], s.join_out)
        if s.others:
            insts = [instance_of(self.tables, r, self.tile_table) for r in s.others]
            s.batch.update(insts)
            s.batch.launch()
        s.event = torch.cuda.Event()
        s.event.record(s.stream)
        s.reqs, s.busy = reqs, True
        self.launches += 1

    def _results(self, s: Slot) -> None:
        """Fills the results of a finished slot's requests (an overflowed
        instance or a shared join over repeated keys is rerun exactly)."""
        if s.lone is not None:
            r = s.lone
            s.engine.ctx.call("bo_check_errors")
            if r.kind == N.BATCH_SCAN_AGG:
                ng = r.params["n_flag_a"] * r.params["n_flag_b"]
                host = s.q1_out[: ng * C.sizeof(N.Q1Agg)].cpu().numpy().tobytes()
                aggs = (N.Q1Agg * ng).from_buffer_copy(host)
                r.result = {"kind": "scan_agg", "groups": [aggs[g].as_dict() for g in range(ng)], "reruns": 0}
            else:
                d = N.JoinResult.from_buffer_copy(s.join_out[: C.sizeof(N.JoinResult)].cpu().numpy().tobytes()).as_dict()
                if d["overflowed"]:  # predicted too few qualifying rows: the exact form
                    d = B.solo_result(s.engine, instance_of(self.tables, r))
                    d["reruns"] = 1
                d["kind"] = "join"
                r.result = d
            return
        if s.others:
            for r, x in zip(s.others, s.batch.results()):
                r.result = x
        if s.gbs:
            s.engine.ctx.call("bo_check_errors")  # device errors of the slot's pipelines (the batch's are read above)
            host = s.gb_out[: len(s.gbs) * C.sizeof(N.GbResult)].cpu().numpy().tobytes()
            for i, r in enumerate(s.gbs):
                d = N.GbResult.from_buffer_copy(host[i * C.sizeof(N.GbResult):]).as_dict()
                if d["overflowed"]:  # predicted too few groups: the exact form
                    d = B.solo_result(s.engine, instance_of(self.tables, r))
                    d["reruns"] = 1
                d["kind"] = "groupby"
                r.result = d
        if s.joins:
            s.engine.ctx.call("bo_check_errors")  # device errors of the shared joins (the batch's are read above)
            host = s.join_out[: len(s.joins) * C.sizeof(N.JoinResult)].cpu().numpy().tobytes()
            for i, r in enumerate(s.joins):
                d = N.JoinResult.from_buffer_copy(host[i * C.sizeof(N.JoinResult):]).as_dict()
                if d["overflowed"]:
                    d = B.solo_result(s.engine, instance_of(self.tables, r))
                    d["reruns"] = 1
                d["kind"] = "join"
                r.result = d

    def serve(self, requests: list[Request]) -> list[Request]:
        """Runs the arrival stream in real time; fills each request's result
        and completion time."""
        pending: deque = deque()
        foot: dict = {}
        n, i, finished = len(requests), 0, 0
        t0 = time.perf_counter()
        while finished < n:
            now = time.perf_counter() - t0
            arrived = []
            while i < n and requests[i].arrival <= now:
                arrived.append(requests[i])
                i += 1
            if arrived:
                # Shared joins size their tables from exact counts (the lone one's and the
                # shared pass's count kernel): only batch-instance joins use a prediction.
                predict_requests(self.tables, arrived, None if self.shared else self.join_sizer, self.gb_sizer)
                for r in arrived:
                    foot[r.rid] = self._footprint(r)
                    pending.append(r)
            for s in self.slots:
                if s.busy and s.event.query():
                    self._results(s)
                    t_done = time.perf_counter() - t0
                    for r in s.reqs:
                        r.done = t_done
                    finished += len(s.reqs)
                    s.reqs, s.busy = [], False
            running = sum(1 for s in self.slots if s.busy)
            for s in self.slots:
                if not s.busy and pending:
                    waited = (time.perf_counter() - t0 - pending[0].arrival) * 1e3
                    if running and len(pending) < self.spill_queue and waited < self.spill_wait_ms:
                        break  # the running slot keeps the GPU a little longer
                    running += 1
                    kind = next_kind(pending, self.policy, waited, self.max_wait_ms)
                    mb = 1 if len(pending) < self.batch_from else self.max_batch
                    reqs = admit(pending, foot, mb, self.pool_bytes, self.max_items, kind)
                    tb = sum(foot[r.rid][0] for r in reqs)
                    if tb > self.pool_bytes:  # a single request above the pool: upper-bound tables do not fit
                        raise RuntimeError(f"request {reqs[0].rid} needs {tb} bytes of tables, slot holds "
                                           f"{self.pool_bytes}")
                    self._launch(s, reqs)
        return requests


def serve_one_per_launch(engine, tables: ServingTables, requests: list[Request]) -> list[Request]:
    """Baseline: each request alone, in arrival order, plain exact-count form."""
    t0 = time.perf_counter()
    for r in requests:
        while time.perf_counter() - t0 < r.arrival:
            pass
        r.result = B.solo_result(engine, instance_of(tables, r))
        r.done = time.perf_counter() - t0
    return requests


def latency_stats(requests: list[Request]) -> dict:
    lat = np.array([r.latency_ms for r in requests])
    span = max(r.done for r in requests) - min(r.arrival for r in requests)
    return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "p99_9_ms": float(np.percentile(lat, 99.9)), "mean_ms": float(lat.mean()),
            "qps": len(requests) / span if span > 0 else math.inf, "requests": len(requests)}
