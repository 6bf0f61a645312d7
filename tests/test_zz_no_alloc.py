"""The allocation-free scan / group-aggregate entry point.

bo_q1_fact_device_noalloc serves callers that may not allocate device memory
when they run a query -- a host process whose memory manager owns every device
allocation, a plugin that is not allowed to call cudaMalloc, or a path that
must not risk the device-wide synchronisation cudaMalloc / cudaFree can cause.
Its scratch is a fixed device array inside the library.  These tests call it
through the C ABI and check it against the regular entry point
(bo_q1_fact_device) on two calls in a row, for a 3 x 2 and a 2 x 4 group
domain (the two kernel instantiations), and against the CPU oracle; results
are exact integers, so the comparison is equality.  This file is named to be
collected last.
"""
import ctypes as C

import numpy as np
import pytest

from bespokeolap_artifacts_b200 import datagen as dg
from bespokeolap_artifacts_b200 import native as N

pytestmark = pytest.mark.gpu


def _records(t, n_groups):
    host = t.cpu().numpy().tobytes()
    recs = (N.Q1Agg * n_groups).from_buffer_copy(host[: n_groups * C.sizeof(N.Q1Agg)])
    return [r.as_dict() for r in recs]


def _fact(n, seed, nfa, nfb):
    t = dg.gen_fact(n, seed)
    if (nfa, nfb) != (3, 2):  # redraw the group codes over the wider domain
        rng = np.random.default_rng(seed + 1000)
        t.flag_a = rng.integers(0, nfa, size=n, dtype=np.uint8)
        t.flag_b = rng.integers(0, nfb, size=n, dtype=np.uint8)
        t.n_flag_a, t.n_flag_b = nfa, nfb
    return t


@pytest.mark.parametrize("nfa,nfb", [(3, 2), (2, 4)])
def test_no_alloc_matches_regular_entry_point_twice(engine, torch_cuda, nfa, nfb):
    torch = torch_cuda
    lib = N.lib()
    stream = torch.cuda.Stream()
    engine.set_stream(stream.cuda_stream)
    ng = nfa * nfb
    try:
        for seed, n in ((31, 1_000_003), (32, 250_001)):  # two calls in a row, different inputs
            t = _fact(n, seed, nfa, nfb)
            cols = [torch.from_numpy(np.ascontiguousarray(c)).cuda() for c in t.columns()]
            fc = N.FactCols(*[c.data_ptr() for c in cols], n)
            out_regular = torch.zeros(N.Q1_MAX_GROUPS * C.sizeof(N.Q1Agg), dtype=torch.uint8, device="cuda")
            out_noalloc = torch.zeros_like(out_regular)
            status = torch.zeros(1, dtype=torch.int32, device="cuda")
            engine.q1_fact_device(cols, n, dg.Q1_CUTOFF, nfa, nfb, out_regular)
            rc = lib.bo_q1_fact_device_noalloc(C.byref(fc), dg.Q1_CUTOFF, nfa, nfb,
                                               C.c_void_p(out_noalloc.data_ptr()), C.c_void_p(status.data_ptr()),
                                               C.c_void_p(stream.cuda_stream))
            assert rc == N.BO_OK
            stream.synchronize()
            assert int(status.item()) == 0
            assert _records(out_noalloc, ng) == _records(out_regular, ng)
    finally:
        engine.set_stream(None)


def test_no_alloc_matches_oracle(torch_cuda):
    torch = torch_cuda
    from oracle import oracle as O

    lib = N.lib()
    stream = torch.cuda.Stream()
    for nfa, nfb in ((3, 2), (2, 4)):
        t = _fact(500_009, 41, nfa, nfb)
        cols = [torch.from_numpy(np.ascontiguousarray(c)).cuda() for c in t.columns()]
        fc = N.FactCols(*[c.data_ptr() for c in cols], t.n_rows)
        out = torch.zeros(N.Q1_MAX_GROUPS * C.sizeof(N.Q1Agg), dtype=torch.uint8, device="cuda")
        status = torch.zeros(1, dtype=torch.int32, device="cuda")
        rc = lib.bo_q1_fact_device_noalloc(C.byref(fc), dg.Q1_CUTOFF, nfa, nfb, C.c_void_p(out.data_ptr()),
                                           C.c_void_p(status.data_ptr()), C.c_void_p(stream.cuda_stream))
        assert rc == N.BO_OK
        stream.synchronize()
        assert int(status.item()) == 0
        want, orc = O.q1_fact(t, dg.Q1_CUTOFF)
        assert orc == 0
        assert _records(out, nfa * nfb) == want


def test_no_alloc_rejects_group_domain_beyond_its_scratch(torch_cuda):
    torch = torch_cuda
    lib = N.lib()
    t = dg.gen_fact(1000, 33)
    cols = [torch.from_numpy(np.ascontiguousarray(c)).cuda() for c in t.columns()]
    fc = N.FactCols(*[c.data_ptr() for c in cols], 1000)
    out = torch.zeros(16 * C.sizeof(N.Q1Agg), dtype=torch.uint8, device="cuda")
    rc = lib.bo_q1_fact_device_noalloc(C.byref(fc), dg.Q1_CUTOFF, 3, 3, C.c_void_p(out.data_ptr()), None, None)
    assert rc == -1  # BO_ERR_INVALID: 9 groups exceed the fixed scratch
