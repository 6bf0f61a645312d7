"""Learned sizing: the MLP that presizes hash tables and output buffers.

The network (``bo_mlp`` in ``csrc/mlp.cu``: n_features -> 64 -> 64 -> 64 ->
n_outputs, FP32, ReLU) is trained on the GPU by the library's own forward /
backward / Adam kernels, on (features, exact count) pairs that the plain GPU
pipeline produces on seeded tables.  Features are predicate constants plus
per-column sketches (``bo_sketch_i32`` / ``bo_histogram_small``: min, max, a
64-bin equi-width histogram, HyperLogLog distinct estimates, exact histograms
of small domains).  Targets are log1p(count).

The prediction only sizes: the exact-count path stays the fallback (a presized
table that overflows is rerun exactly) and the judge (q-error is reported), so
no answer depends on it.  No reference counterpart exists -- the reference
sizes its dense arrays exactly (bespoke_tpch/query_q3.cpp:178-180).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import native as N

LOG_SCALE = 16.0


class Mlp:
    """One ``bo_mlp`` model bound to an engine context."""

    def __init__(self, ctx: N.Context, n_features: int, n_outputs: int, seed: int = 0):
        self.ctx = ctx
        self.F, self.O = n_features, n_outputs
        h = C.c_void_p()
        ctx.check(ctx._lib.bo_mlp_create(ctx.handle, n_features, n_outputs, seed, C.byref(h)), "bo_mlp_create")
        self.handle = h
        self.P = ctx._lib.bo_mlp_num_params(h)

    def close(self):
        if getattr(self, "handle", None):
            self.ctx._lib.bo_mlp_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_params(self) -> np.ndarray:
        out = np.empty(self.P, np.float32)
        self.ctx.call("bo_mlp_get_params", self.handle, C.c_void_p(out.ctypes.data))
        return out

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.shape == (self.P,)
        self.ctx.call("bo_mlp_set_params", self.handle, C.c_void_p(p.ctypes.data))

    def train(self, x: np.ndarray, t: np.ndarray, epochs: int = 2000, lr: float = 3e-3) -> float:
        """Full-batch Adam on host arrays (copied to the device once)."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        loss = C.c_float()
        self.ctx.call("bo_mlp_train_host", self.handle, C.c_void_p(x.ctypes.data), C.c_void_p(t.ctypes.data),
                      x.shape[0], epochs, lr, C.byref(loss))
        return float(loss.value)

    def gradients(self, x_dev, t_dev, n: int, grad_dev, loss_dev) -> None:
        self.ctx.call("bo_mlp_gradients_device", self.handle, C.c_void_p(N.ptr(x_dev)), C.c_void_p(N.ptr(t_dev)),
                      n, C.c_void_p(N.ptr(grad_dev)), C.c_void_p(N.ptr(loss_dev)))

    def infer_device(self, x_dev, n: int, y_dev) -> None:
        self.ctx.call("bo_mlp_infer_device", self.handle, C.c_void_p(N.ptr(x_dev)), n, C.c_void_p(N.ptr(y_dev)))

    def predict_counts_device(self, features: np.ndarray, counts_dev, log_dev=None) -> None:
        """One feature vector (passed to the kernel by value) -> device counts."""
        f = np.ascontiguousarray(features, dtype=np.float32)
        assert f.shape == (self.F,)
        self.ctx.call("bo_mlp_predict_counts", self.handle, C.c_void_p(f.ctypes.data), C.c_void_p(N.ptr(counts_dev)),
                      C.c_void_p(N.ptr(log_dev) if log_dev is not None else 0))


# ------------------------------------------------------------------ sketches --
@dataclass
class IntSketch:
    n: int
    min: int
    max: int
    hist: np.ndarray       # 64 equi-width bins over [min, max]
    distinct: float

    def frac_below(self, v: int) -> float:
        """Estimated fraction of rows with value < v (uniform within a bin)."""
        if self.n == 0:
            return 0.0
        if v <= self.min:
            return 0.0
        if v > self.max:
            return 1.0
        span = self.max - self.min + 1
        pos = (v - self.min) * len(self.hist) / span
        b = int(pos)
        below = float(self.hist[:b].sum()) + float(self.hist[b]) * (pos - b) if b < len(self.hist) else float(
            self.hist.sum())
        return below / self.n

    def frac_between(self, lo: int, hi: int) -> float:
        """Estimated fraction with lo <= value <= hi."""
        return max(0.0, self.frac_below(hi + 1) - self.frac_below(lo))


def sketch_i32(ctx: N.Context, col_dev, n: int) -> IntSketch:
    s = N.Sketch()
    ctx.call("bo_sketch_i32", C.c_void_p(N.ptr(col_dev)), n, C.byref(s))
    return IntSketch(s.n, s.min, s.max, np.array(s.hist[:], dtype=np.int64), s.distinct_estimate)


def histogram_small(ctx: N.Context, col_dev, elem_bytes: int, n: int, domain: int) -> np.ndarray:
    out = np.zeros(domain, np.int64)
    ctx.call("bo_histogram_small", C.c_void_p(N.ptr(col_dev)), elem_bytes, n, domain, C.c_void_p(out.ctypes.data))
    return out


# --------------------------------------------------------- join build sizing --
JOIN_FEATURES = 8


@dataclass
class JoinTableStats:
    """Load-time statistics of a join build side (computed once per table)."""
    n: int
    date: IntSketch
    key: IntSketch
    seg_hist: np.ndarray   # 256 counts


def join_table_stats(ctx: N.Context, key_dev, date_dev, seg_dev, n: int) -> JoinTableStats:
    return JoinTableStats(n, sketch_i32(ctx, date_dev, n), sketch_i32(ctx, key_dev, n),
                          histogram_small(ctx, seg_dev, 1, n, 256))


def join_independence_estimate(st: JoinTableStats, date_lt: int, seg_eq: int) -> float:
    """The classic estimate: n * sel(date) * sel(segment), columns independent."""
    if st.n == 0:
        return 0.0
    return st.n * st.date.frac_below(date_lt) * (st.seg_hist[seg_eq] / st.n)


def join_features(st: JoinTableStats, date_lt: int, seg_eq: int) -> np.ndarray:
    n = max(st.n, 1)
    fd = st.date.frac_below(date_lt)
    fs = st.seg_hist[seg_eq] / n
    span = max(st.date.max - st.date.min + 1, 1)
    return np.array([
        math.log1p(st.n) / LOG_SCALE,
        fd,
        min(max((date_lt - st.date.min) / span, -0.5), 1.5),
        fs,
        math.log1p(st.n * fd * fs) / LOG_SCALE,
        math.log1p(st.key.distinct) / LOG_SCALE,
        fd * fs,
        float(np.count_nonzero(st.seg_hist)) / 16.0,
    ], dtype=np.float32)


def gen_join_training_table(rng: np.random.Generator, n: int) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """A seeded build side with varied shape: uniform or skewed dates, uniform or
    skewed segments, and (half the time) segments correlated with dates so the
    independence estimate is wrong."""
    from .datagen import DATE_HI, DATE_LO

    key = rng.permutation(np.arange(1, n + 1, dtype=np.int32))
    span = DATE_HI - DATE_LO
    if rng.random() < 0.5:
        date = rng.integers(DATE_LO, DATE_HI, size=n, endpoint=True, dtype=np.int32)
    else:
        date = (DATE_LO + span * rng.beta(rng.uniform(0.5, 3), rng.uniform(0.5, 3), size=n)).astype(np.int32)
    k = int(rng.integers(2, 9))
    if rng.random() < 0.5:
        seg = rng.integers(0, k, size=n, dtype=np.uint8)
    else:
        w = np.arange(1, k + 1, dtype=np.float64) ** -rng.uniform(0.5, 2.0)
        seg = rng.choice(k, size=n, p=w / w.sum()).astype(np.uint8)
    if rng.random() < 0.5:  # correlate segment with date
        bucket = ((date - DATE_LO) * k // (span + 1)).astype(np.int64)
        noisy = rng.random(n) < rng.uniform(0.0, 0.5)
        seg = np.where(noisy, seg, bucket % k).astype(np.uint8)
    return key, date, seg


def gen_join_training_table_device(rng: np.random.Generator, n: int):
    """The same family of build sides as gen_join_training_table, generated on
    the device (seeded from `rng`) so that tables of tens of millions of rows
    cost milliseconds."""
    import torch

    from .datagen import DATE_HI, DATE_LO

    g = torch.Generator(device="cuda")
    g.manual_seed(int(rng.integers(1 << 62)))
    key = (torch.randperm(n, generator=g, device="cuda") + 1).to(torch.int32)
    span = DATE_HI - DATE_LO
    if rng.random() < 0.5:
        date = torch.randint(DATE_LO, DATE_HI + 1, (n,), generator=g, device="cuda", dtype=torch.int32)
    else:
        a, b = float(rng.uniform(0.5, 3)), float(rng.uniform(0.5, 3))
        # Beta(a, b) as X / (X + Y) with X ~ Gamma(a), Y ~ Gamma(b) (torch's gamma sampler takes no generator,
        # so the uniform draws are transformed instead: inverse-CDF of the beta is not closed-form, the
        # gamma route is seeded through the global device generator below).
        torch.cuda.manual_seed(int(rng.integers(1 << 62)))
        x = torch._standard_gamma(torch.full((n,), a, device="cuda"))
        y = torch._standard_gamma(torch.full((n,), b, device="cuda"))
        date = (DATE_LO + span * (x / (x + y))).to(torch.int32)
    k = int(rng.integers(2, 9))
    if rng.random() < 0.5:
        seg = torch.randint(0, k, (n,), generator=g, device="cuda", dtype=torch.int32)
    else:
        w = torch.arange(1, k + 1, dtype=torch.float64, device="cuda").pow(-float(rng.uniform(0.5, 2.0)))
        seg = torch.multinomial(w, n, replacement=True, generator=g).to(torch.int32)
    if rng.random() < 0.5:  # correlate segment with date
        bucket = ((date.to(torch.int64) - DATE_LO) * k // (span + 1)) % k
        noisy = torch.rand(n, generator=g, device="cuda") < float(rng.uniform(0.0, 0.5))
        seg = torch.where(noisy, seg, bucket.to(torch.int32))
    return key, date, seg.to(torch.uint8)


def make_join_training_set(engine, n_tables: int = 24, preds_per_table: int = 40, seed: int = 1234,
                           n_min: int = 20_000, n_max: int = 2_000_000, device_gen: bool = False):
    """(features, log1p(exact qualifying rows), independence estimates): the
    exact counts come from the plain GPU pipeline's count kernel (K7).
    device_gen draws the tables on the device (for large n_max)."""
    import torch

    from .datagen import DATE_HI, DATE_LO

    rng = np.random.default_rng(seed)
    xs, ts, naive = [], [], []
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    for _ in range(n_tables):
        n = int(math.exp(rng.uniform(math.log(n_min), math.log(n_max))))
        if device_gen:
            dk, dd, ds = gen_join_training_table_device(rng, n)
        else:
            key, date, seg = gen_join_training_table(rng, n)
            dk, dd, ds = (torch.from_numpy(a).cuda() for a in (key, date, seg))
        st = join_table_stats(engine.ctx, dk, dd, ds, n)
        for _ in range(preds_per_table):
            d = int(rng.integers(DATE_LO, DATE_HI + 2))
            s = int(rng.integers(0, 8))
            engine.join_count_device((dk, dd, ds), n, d, s, cnt)
            engine.synchronize()
            c = int(cnt.item())
            xs.append(join_features(st, d, s))
            ts.append([math.log1p(c)])
            naive.append(join_independence_estimate(st, d, s))
    return np.stack(xs), np.array(ts, np.float32), np.array(naive)


def q_error(pred, true) -> np.ndarray:
    """max(p/t, t/p) with both counts floored at 1."""
    p = np.maximum(np.asarray(pred, dtype=np.float64), 1.0)
    t = np.maximum(np.asarray(true, dtype=np.float64), 1.0)
    return np.maximum(p / t, t / p)


def split_holdout(n: int, frac: float = 0.2, seed: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """Seeded (train, holdout) index split."""
    idx = np.random.default_rng(seed).permutation(n)
    k = int(round(n * (1.0 - frac)))
    return idx[:k], idx[k:]


def calibrate_margin(mlp: Mlp, pred_counts: np.ndarray, exact_counts: np.ndarray, quantile: float = 0.9,
                     output: int = 0) -> float:
    """Safety margin from held-out data: the `quantile` of exact / predicted
    (at least 1).  The margin is folded into the network itself -- log(margin)
    is added to the output's final bias, so every later prediction (host or
    device) comes out about `margin` times larger.  A table sized from an
    under-prediction runs at high load (long probe chains) or overflows and is
    rerun, while an over-prediction only costs memory, so sizing from an upper
    quantile is the cheaper side to err on."""
    ratio = np.maximum(np.asarray(exact_counts, np.float64), 1.0) / np.maximum(np.asarray(pred_counts, np.float64), 1.0)
    m = float(max(1.0, np.quantile(ratio, quantile))) if len(ratio) else 1.0
    p = mlp.get_params()
    p[len(p) - mlp.O + output] += math.log(m)
    mlp.set_params(p)
    return m


class JoinSizer:
    """Trained join-build sizer: features -> predicted qualifying build rows,
    written on the device where the presized join reads it."""

    def __init__(self, engine, seed: int = 7):
        self.engine = engine
        self.mlp = Mlp(engine.ctx, JOIN_FEATURES, 1, seed)
        self.margin = 1.0

    def calibrate(self, x, t, quantile: float = 0.9) -> float:
        """Scales later predictions by the held-out quantile of exact / predicted."""
        self.margin = calibrate_margin(self.mlp, self.predict_host(x), np.expm1(np.asarray(t)[:, 0]), quantile)
        return self.margin

    def fit(self, x, t, epochs: int = 3000, lr: float = 2e-3) -> float:
        return self.mlp.train(x, t, epochs, lr)

    def predict_host(self, x: np.ndarray) -> np.ndarray:
        """Batch inference on the device (used for evaluation), counts on host."""
        import torch

        xd = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float32)).cuda()
        yd = torch.empty((x.shape[0], 1), dtype=torch.float32, device="cuda")
        self.mlp.infer_device(xd, x.shape[0], yd)
        self.engine.synchronize()
        return np.expm1(yd.cpu().numpy()[:, 0].astype(np.float64)).clip(min=0)

    def predict_device(self, features: np.ndarray, counts_dev) -> None:
        self.mlp.predict_counts_device(features, counts_dev)

    def join_device(self, features: np.ndarray, build, probe, n_build: int, n_probe: int, date_lt: int,
                    seg_eq: int, out_dev, pred_dev=None) -> None:
        """The learned join in one call (bo_join_learned_device): the MLP
        prediction is folded into the table's init kernel."""
        f = np.ascontiguousarray(features, dtype=np.float32)
        b = N.JoinBuildCols(*[N.ptr(c) for c in build], n_build)
        p = N.JoinProbeCols(*[N.ptr(c) for c in probe], n_probe)
        self.engine.ctx.call("bo_join_learned_device", self.mlp.handle, C.c_void_p(f.ctypes.data), C.byref(b),
                             C.byref(p), C.byref(N.JoinParams(date_lt, seg_eq)), C.c_void_p(N.ptr(out_dev)),
                             C.c_void_p(N.ptr(pred_dev) if pred_dev is not None else 0))

    def join(self, features: np.ndarray, build, probe, n_build: int, n_probe: int, date_lt: int,
             seg_eq: int) -> dict:
        """bo_join_learned: synchronous, exact rerun if the table overflowed."""
        f = np.ascontiguousarray(features, dtype=np.float32)
        b = N.JoinBuildCols(*[N.ptr(c) for c in build], n_build)
        p = N.JoinProbeCols(*[N.ptr(c) for c in probe], n_probe)
        out = N.JoinResult()
        self.engine.ctx.call("bo_join_learned", self.mlp.handle, C.c_void_p(f.ctypes.data), C.byref(b), C.byref(p),
                             C.byref(N.JoinParams(date_lt, seg_eq)), C.byref(out))
        return out.as_dict()

    # Fan-out of the radix-partitioned join from the predicted qualifying build
    # rows: one pass while the single-pass table (4 slots of 8 bytes per
    # row) fits in half the L2, else partitions of about 4096 keys (half of a
    # partition's 8192-slot shared-memory table).
    PART_KEYS = 4096

    @classmethod
    def fanout(cls, predicted_rows: float, l2_bytes: int = 126 << 20) -> int:
        """log2 of the partition count for a predicted qualifying-row count (0 = single pass)."""
        r = max(0.0, float(predicted_rows))
        if r * 4 * 8 <= l2_bytes / 2:
            return 0
        return int(min(N.JOIN_MAX_LOG2_PARTITIONS, max(1, math.ceil(math.log2(r / cls.PART_KEYS)))))


# ------------------------------------------------------ group-by sizing -----
GB_FEATURES = 12
CAT_DOMAIN = 4096


@dataclass
class GroupByTableStats:
    """Load-time statistics of the three group-by inputs."""
    n_a: int
    n_b: int
    n_c: int
    year: IntSketch
    cat_hist: np.ndarray   # exact counts of category codes < CAT_DOMAIN
    b_a: IntSketch         # HLL distinct of B.a_id
    b_c: IntSketch         # HLL distinct of B.c_id


def groupby_table_stats(ctx: N.Context, dev: dict, n_a: int, n_b: int, n_c: int) -> GroupByTableStats:
    return GroupByTableStats(
        n_a, n_b, n_c, sketch_i32(ctx, dev["c_year"], n_c), histogram_small(ctx, dev["c_cat"], 2, n_c, CAT_DOMAIN),
        sketch_i32(ctx, dev["b_a"], n_b), sketch_i32(ctx, dev["b_c"], n_b))


def groupby_naive(st: GroupByTableStats, cat_set, year_lo: int, year_hi: int) -> tuple[float, float]:
    """Independence / uniformity estimates: joined rows = n_b * sel(C), groups =
    distinct a_ids that see at least one joining row (rows spread evenly)."""
    if st.n_c == 0 or st.n_b == 0:
        return 0.0, 0.0
    f_cat = float(st.cat_hist[np.asarray(cat_set, dtype=np.int64)].sum()) / st.n_c
    f_c = f_cat * st.year.frac_between(year_lo, year_hi)
    joined = st.n_b * f_c
    d_a = max(st.b_a.distinct, 1.0)
    per_a = st.n_b / d_a
    groups = d_a * (1.0 - (1.0 - min(f_c, 1.0)) ** per_a)
    return groups, joined


def groupby_features(st: GroupByTableStats, cat_set, year_lo: int, year_hi: int) -> np.ndarray:
    f_cat = float(st.cat_hist[np.asarray(cat_set, dtype=np.int64)].sum()) / max(st.n_c, 1)
    f_year = st.year.frac_between(year_lo, year_hi)
    groups, joined = groupby_naive(st, cat_set, year_lo, year_hi)
    lg = lambda v: math.log1p(max(v, 0.0)) / LOG_SCALE  # noqa: E731
    return np.array([
        lg(st.n_a), lg(st.n_b), lg(st.n_c), f_cat, f_year, f_cat * f_year,
        lg(st.b_a.distinct), lg(st.b_c.distinct), st.b_a.distinct / max(st.n_b, 1),
        st.b_c.distinct / max(st.n_b, 1), lg(groups), lg(joined),
    ], dtype=np.float32)


def make_groupby_training_set(engine, n_tables: int = 16, preds_per_table: int = 30, seed: int = 77,
                              nb_min: int = 100_000, nb_max: int = 4_000_000, device_gen: bool = False):
    """(features, [log1p(groups), log1p(joined)], naive estimates): exact targets
    from the plain GPU pipeline's pre-pass (bo_groupby_distinct_device).
    device_gen draws the tables on the device (for large nb_max)."""
    import torch

    from .datagen import GroupByInput, gen_groupby

    rng = np.random.default_rng(seed)
    xs, ts, naive = [], [], []
    out = torch.zeros(2, dtype=torch.int64, device="cuda")
    for _ in range(n_tables):
        n_b = int(math.exp(rng.uniform(math.log(nb_min), math.log(nb_max))))
        n_a = max(1000, int(n_b * rng.uniform(0.02, 0.2)))
        n_c = max(1000, int(n_b * rng.uniform(0.05, 0.3)))
        s_a, s_c = float(rng.uniform(0.7, 1.4)), float(rng.uniform(0.5, 1.2))
        tseed = int(rng.integers(1 << 30))
        if device_gen:
            from .batching import groupby_tables_device

            dev = groupby_tables_device(n_a, n_b, n_c, tseed, s_a, s_c)
            g = GroupByInput(np.zeros(n_a, np.int32), np.zeros(0, np.int32), np.zeros(0, np.int32),
                             np.zeros(0, np.uint16), np.zeros(0, np.int32), np.zeros(0, np.uint16), 0, 0)
        else:
            g = gen_groupby(n_a, n_b, n_c, seed=tseed, s_a=s_a, s_c=s_c)
            dev = engine.groupby_to_device(g)
        st = groupby_table_stats(engine.ctx, dev, n_a, n_b, n_c)
        for _ in range(preds_per_table):
            k = int(rng.integers(1, 17))
            cats = np.sort(rng.choice(113, size=k, replace=False)).astype(np.uint16)
            lo = int(rng.integers(1900, 2021))
            hi = int(min(2020, lo + rng.integers(0, 60)))
            q = GroupByInput(g.a_ids, g.b_a, g.b_c, g.c_cat, g.c_year, cats, lo, hi, 10, g.seed)
            engine.groupby_distinct_device(dev, q, out)
            engine.synchronize()
            groups, joined = (int(v) for v in out.tolist())
            xs.append(groupby_features(st, cats, lo, hi))
            ts.append([math.log1p(groups), math.log1p(joined)])
            naive.append(groupby_naive(st, cats, lo, hi))
        del dev
    return np.stack(xs), np.array(ts, np.float32), np.array(naive)


class GroupBySizer:
    """Trained group-table sizer: features -> predicted (groups, joined rows);
    the group count is written on the device for the presized group-by."""

    def __init__(self, engine, seed: int = 9):
        self.engine = engine
        self.mlp = Mlp(engine.ctx, GB_FEATURES, 2, seed)
        self.margin = 1.0

    def calibrate(self, x, t, quantile: float = 0.9) -> float:
        """Scales later group-count predictions by the held-out quantile of
        exact / predicted."""
        self.margin = calibrate_margin(self.mlp, self.predict_host(x)[:, 0], np.expm1(np.asarray(t)[:, 0]), quantile)
        return self.margin

    def fit(self, x, t, epochs: int = 3000, lr: float = 2e-3) -> float:
        return self.mlp.train(x, t, epochs, lr)

    def predict_host(self, x: np.ndarray) -> np.ndarray:
        import torch

        xd = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float32)).cuda()
        yd = torch.empty((x.shape[0], 2), dtype=torch.float32, device="cuda")
        self.mlp.infer_device(xd, x.shape[0], yd)
        self.engine.synchronize()
        return np.expm1(yd.cpu().numpy().astype(np.float64)).clip(min=0)

    def predict_device(self, features: np.ndarray, counts_dev) -> None:
        """counts_dev[0] = predicted groups, counts_dev[1] = predicted joined rows."""
        self.mlp.predict_counts_device(features, counts_dev)

    # Fan-out of the radix-partitioned group-by from the predicted group count:
    # one pass while the single-pass table (2.5 slots of 12 bytes per group)
    # fits in half the L2, else partitions of about 4096 groups (half of a
    # partition's 8192-slot shared-memory table).
    PART_GROUPS = 4096

    @classmethod
    def fanout(cls, predicted_groups: float, l2_bytes: int = 126 << 20) -> int:
        """log2 of the partition count for a predicted group count (0 = single pass)."""
        g = max(0.0, float(predicted_groups))
        if g * 2.5 * 12 <= l2_bytes / 2:
            return 0
        return int(min(N.GB_MAX_LOG2_PARTITIONS, max(1, math.ceil(math.log2(g / cls.PART_GROUPS)))))
