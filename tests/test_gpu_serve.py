"""Batched execution and the serving loop on the GPU: every request of a mixed batch equals
its oracle result and its solo execution; a request that fails reports only its own status;
served results are the same alone and in the mix under continuous batching; admission by
predicted footprint rejects what can never fit and serialises what does not fit now."""
import ctypes as C

import pytest

from gpudbmetalbenchmark_b200 import capi
from gpudbmetalbenchmark_b200.engine import q1_to_dict, q3_to_list
from gpudbmetalbenchmark_b200.serve import Server, Workload, open_loop

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small(engine):
    return Workload(engine, scan_rows=(100_003, 1_000_003), q3=(3000, 30_000, 120_000), q9=(4000, 400, 20_000, 100_000))


def test_mixed_batch_matches_oracle(engine, orc):
    li = orc.lineitem(200_003, seed=5)
    t = engine.upload("lineitem", li)
    s = t.lineitem()
    cu_, od_, l3 = orc.q3_tables(3000, 30_000, 120_000, 6)
    q3t = capi.Q3Tables(engine.upload("customer", cu_).struct(), engine.upload("orders", od_).struct(),
                        engine.upload("lineitem", l3).lineitem())
    reqs = (capi.Request * 7)()
    outs = []
    # Q6 over uneven row ranges, Q1 over all rows and a range, Q3 global and radix, a bad request
    ranges = [(0, 0), (17, 150_000), (150_000, 200_003)]
    for i, (b, e) in enumerate(ranges):
        reqs[i].pipeline = capi.PIPE_Q6
        reqs[i].li = C.pointer(s)
        reqs[i].row_begin, reqs[i].row_end = b, e
        reqs[i].q6 = capi.Q6Params(300 + 100 * i, 900, 2, 8, 40)
        o = capi.Q6Result()
        outs.append(o)
        reqs[i].q6_out = C.pointer(o)
    o1 = capi.Q1Result()
    reqs[3].pipeline, reqs[3].li, reqs[3].q1, reqs[3].q1_out = capi.PIPE_Q1, C.pointer(s), capi.Q1Params(2000, 0), C.pointer(o1)
    o3a, o3b = capi.Q3Result(), capi.Q3Result()
    for j, (o, mode) in enumerate(((o3a, capi.JOIN_GLOBAL), (o3b, capi.JOIN_RADIX))):
        r = reqs[4 + j]
        r.pipeline, r.q3, r.q3_out = capi.PIPE_Q3, C.pointer(q3t), C.pointer(o)
        r.q3p = capi.Q3Params(2, 1500, 800, 12, mode, 0)
    reqs[6].pipeline = 77
    engine._check(engine.lib.gpudb_batch_run(engine.ctx, reqs, 7, None, None))
    for i, (b, e) in enumerate(ranges):
        e = e or 200_003
        sub = {k: v[b:e] for k, v in li.items()}
        assert reqs[i].status == capi.OK
        assert (outs[i].revenue, outs[i].rows_matched) == orc.q6(sub, 300 + 100 * i, 900, 2, 8, 40)
    assert reqs[3].status == capi.OK and q1_to_dict(o1) == orc.q1(li, 2000)
    want3 = orc.q3(cu_, od_, l3, 2, 1500, 800, 12)
    assert q3_to_list(o3a) == want3 and q3_to_list(o3b) == want3
    assert reqs[6].status == capi.E_INVALID


def test_failing_request_does_not_fail_its_batch(engine, orc):
    li = orc.lineitem(50_000, seed=8)
    li["discount"][10] = 500          # outside the exact-arithmetic domain of Q1
    li["ship_date"][10] = 0
    t = engine.upload("lineitem", li)
    s = t.lineitem()
    reqs = (capi.Request * 2)()
    o1, o6 = capi.Q1Result(), capi.Q6Result()
    reqs[0].pipeline, reqs[0].li, reqs[0].q1, reqs[0].q1_out = capi.PIPE_Q1, C.pointer(s), capi.Q1Params(2436, 0), C.pointer(o1)
    reqs[1].pipeline, reqs[1].li, reqs[1].q6, reqs[1].q6_out = (capi.PIPE_Q6, C.pointer(s), capi.Q6Params(0, 2527, 0, 1000, 99),
                                                                C.pointer(o6))
    engine._check(engine.lib.gpudb_batch_run(engine.ctx, reqs, 2, None, None))
    assert reqs[0].status == capi.E_INVALID
    assert reqs[1].status == capi.OK and (o6.revenue, o6.rows_matched) == orc.q6(li, 0, 2527, 0, 1000, 99)


def test_many_scans_in_one_batch(engine, small):
    jobs = [j for j in small.jobs(1500, seed=3) if j.kind in (capi.PIPE_Q6, capi.PIPE_Q1)]
    solo = small.solo_results(jobs)
    for j in jobs:
        j.out.__init__()   # clear results
    arr = (capi.Request * len(jobs))(*[j.req for j in jobs])
    engine._check(engine.lib.gpudb_batch_run(engine.ctx, arr, len(jobs), None, None))
    for k, j in enumerate(jobs):
        assert arr[k].status == capi.OK
        assert j.result() == solo[k]


@pytest.mark.parametrize("no_key_bound", [False, True])
def test_batched_q3_matches_solo(engine, small, no_key_bound):
    """Q3 requests over the same tables run as batched launches (groups of up to 8, so 19
    requests make three groups): each equals the request run alone, for any segment, date
    bounds and k, with and without the orders key bound (order-key bitmaps off)."""
    import random
    rng = random.Random(31 + no_key_bound)
    tables = small.q3
    if no_key_bound:
        od = capi.Orders.from_buffer_copy(tables.od)
        od.key_max = -1
        tables = capi.Q3Tables(tables.cu, od, tables.li)
    jobs = []
    for i in range(19):
        r = capi.Request(pipeline=capi.PIPE_Q3)
        r.q3 = C.pointer(tables)
        seg = rng.choice([0, 1, 1, 4, 7])             # 7: no customer has it
        r.q3p = capi.Q3Params(seg, rng.randrange(-1, 2500), rng.randrange(-1, 2600), rng.choice([1, 3, 10, 64]),
                              capi.JOIN_GLOBAL, 0)
        out = capi.Q3Result()
        r.q3_out = C.pointer(out)
        from gpudbmetalbenchmark_b200.serve import Job
        jobs.append(Job(capi.PIPE_Q3, r, out))
    solo = small.solo_results(jobs)
    for j in jobs:
        j.out.__init__()
    arr = (capi.Request * len(jobs))(*[j.req for j in jobs])
    engine._check(engine.lib.gpudb_batch_run(engine.ctx, arr, len(jobs), None, None))
    for k, j in enumerate(jobs):
        assert arr[k].status == capi.OK
        assert j.result() == solo[k], k


def test_identical_joins_in_one_batch(engine, small):
    """Identical Q3/Q9 requests of one batch run once; every copy gets the full result."""
    base = [j for j in small.jobs(200, seed=23) if j.kind in (capi.PIPE_Q3, capi.PIPE_Q9)][:4]
    jobs = []
    for j in base:   # each request three times, plus a different Q3
        for _ in range(3):
            jobs.append(small.make_like(j))
    solo = small.solo_results(jobs)
    for j in jobs:
        j.out.__init__()
        j.req.q9_groups = 0
    arr = (capi.Request * len(jobs))(*[j.req for j in jobs])
    engine._check(engine.lib.gpudb_batch_run(engine.ctx, arr, len(jobs), None, None))
    for k, j in enumerate(jobs):
        assert arr[k].status == capi.OK
        j.req.q9_groups = arr[k].q9_groups
        assert j.result() == solo[k]


def test_shared_scan_q1_cutoffs_and_q6_mix(engine, orc):
    """One shared pass: Q1 cutoffs that tie, select nothing and select everything, with
    more than one pass's worth of Q6 and Q1 requests over the same rows."""
    li = orc.lineitem(70_001, seed=21)
    s = engine.upload("lineitem", li).lineitem()
    cuts = [-1, 0, 1200, 1200, 2526, 2**31 - 1] + [100 * i for i in range(14)]
    q6s = [(100 * i, 100 * i + 400, i % 11, min(10, i % 11 + 2), 10 + i) for i in range(20)]
    reqs = (capi.Request * (len(cuts) + len(q6s)))()
    o1 = [capi.Q1Result() for _ in cuts]
    o6 = [capi.Q6Result() for _ in q6s]
    for i, c in enumerate(cuts):
        r = reqs[2 * i if i < len(q6s) else len(q6s) + i]
        r.pipeline, r.li, r.q1, r.q1_out = capi.PIPE_Q1, C.pointer(s), capi.Q1Params(c, 0), C.pointer(o1[i])
    taken = {2 * i if i < len(q6s) else len(q6s) + i for i in range(len(cuts))}
    free = [k for k in range(len(reqs)) if k not in taken]
    for i, p in enumerate(q6s):
        r = reqs[free[i]]
        r.pipeline, r.li, r.q6, r.q6_out = capi.PIPE_Q6, C.pointer(s), capi.Q6Params(*p), C.pointer(o6[i])
    engine._check(engine.lib.gpudb_batch_run(engine.ctx, reqs, len(reqs), None, None))
    assert all(r.status == capi.OK for r in reqs)
    for c, o in zip(cuts, o1):
        assert q1_to_dict(o) == orc.q1(li, c), c
    for p, o in zip(q6s, o6):
        assert (o.revenue, o.rows_matched) == orc.q6(li, *p), p


def test_serve_warmup(engine, small):
    jobs = small.jobs(40, seed=17)
    solo = small.solo_results(jobs)
    for j in jobs:
        j.out.__init__()
        j.req.q9_groups = 0
    srv = Server(lanes=3, max_batch=16)
    try:
        srv.warmup(jobs)
        assert [j.result() for j in jobs] == solo
        lat, status, wall = open_loop(srv, small.jobs(100, seed=18), 5000.0, seed=3)
    finally:
        srv.close()
    assert all(s == capi.OK for s in status)


@pytest.mark.parametrize("lanes,max_batch,rate", [(1, 1, 3000.0), (4, 64, 20000.0), (2, 8, 50000.0)])
def test_served_results_same_alone_and_in_the_mix(engine, small, lanes, max_batch, rate):
    jobs = small.jobs(1200, seed=int(rate))
    solo = small.solo_results(jobs)
    for j in jobs:
        j.out.__init__()
        j.req.q9_groups = 0
    srv = Server(lanes=lanes, max_batch=max_batch)
    try:
        lat, status, wall = open_loop(srv, jobs, rate, seed=1)
        st = srv.stats()
    finally:
        srv.close()
    assert all(s == capi.OK for s in status)
    assert [j.result() for j in jobs] == solo
    assert st["completed"] == len(jobs) and st["failed"] == 0
    if max_batch > 1:
        assert st["max_batch_seen"] > 1   # arrivals during running batches were batched


def test_admission_by_footprint(engine, small):
    jobs = small.jobs(300, seed=11)
    q3 = next(j for j in jobs if j.kind == capi.PIPE_Q3)
    fp = engine.lib.gpudb_request_footprint(C.byref(q3.req))
    assert fp > 1 << 20
    srv = Server(lanes=2, max_batch=16, memory_budget=fp // 2)
    try:
        with pytest.raises(capi.GpudbError) as e:
            srv.submit(q3.req)
        assert e.value.code == capi.E_BUSY
    finally:
        srv.close()
    # a budget that admits one join at a time still completes everything, exactly
    solo = small.solo_results(jobs)
    for j in jobs:
        j.out.__init__()
        j.req.q9_groups = 0
    big = max(engine.lib.gpudb_request_footprint(C.byref(j.req)) for j in jobs)
    srv = Server(lanes=3, max_batch=32, memory_budget=big)
    try:
        lat, status, wall = open_loop(srv, jobs, 20000.0, seed=2)
        st = srv.stats()
    finally:
        srv.close()
    assert all(s == capi.OK for s in status)
    assert [j.result() for j in jobs] == solo
    assert st["peak_admitted_bytes"] <= big


@pytest.mark.parametrize("n1,n6", [(1, 1), (1, 2), (1, 4), (1, 5), (2, 1), (2, 2), (2, 6), (3, 4), (4, 9)])
def test_q6_requests_riding_on_a_q1_scan(engine, orc, n1, n6):
    """n1 Q1 requests and n6 Q6 requests over the same rows: a lone Q1 request's kernel also
    evaluates up to four Q6 requests on the rows it reads; other mixes go their own way
    (single-request kernels, or shared passes for more requests); every result equals the
    oracle's."""
    li = orc.lineitem(300_007, seed=31)
    s = engine.upload("lineitem", li).lineitem()
    q6s = [(100 + 300 * i, 900 + 300 * i, i % 5, i % 5 + 4, 20 + 5 * i) for i in range(n6)]
    q6s[-1] = (2000, 1000, 0, 10, 50)   # an empty ship range: nothing matches
    q1s = [1800 - 250 * i for i in range(n1)]
    reqs = (capi.Request * (n1 + n6))()
    o1 = [capi.Q1Result() for _ in q1s]
    for i, le in enumerate(q1s):
        r = reqs[i]
        r.pipeline, r.li, r.q1, r.q1_out = capi.PIPE_Q1, C.pointer(s), capi.Q1Params(le, 0), C.pointer(o1[i])
    o6 = [capi.Q6Result() for _ in q6s]
    for i, p in enumerate(q6s):
        r = reqs[n1 + i]
        r.pipeline, r.li, r.q6, r.q6_out = capi.PIPE_Q6, C.pointer(s), capi.Q6Params(*p), C.pointer(o6[i])
    engine._check(engine.lib.gpudb_batch_run(engine.ctx, reqs, len(reqs), None, None))
    assert all(r.status == capi.OK for r in reqs)
    for le, o in zip(q1s, o1):
        assert q1_to_dict(o) == orc.q1(li, le), le
    for p, o in zip(q6s, o6):
        assert (o.revenue, o.rows_matched) == orc.q6(li, *p), p


def test_heavy_lane_takes_the_large_scans(engine):
    """With a heavy lane, scans of a table over 2^24 rows go to it and everything else to the
    other lanes; every result is the same as alone, and a config with no light lane is refused."""
    wl = Workload(engine, scan_rows=(100_003, 20_000_000), q3=(3000, 30_000, 120_000),
                  q9=(4000, 400, 20_000, 100_000))
    jobs = wl.jobs(600, seed=29)
    solo = wl.solo_results(jobs)
    for j in jobs:
        j.out.__init__()
        j.req.q9_groups = 0
    srv = Server(lanes=3, max_batch=32, heavy_lanes=1)
    try:
        lat, status, wall = open_loop(srv, jobs, 20000.0, seed=2)
        st = srv.stats()
    finally:
        srv.close()
    assert all(s == capi.OK for s in status)
    assert [j.result() for j in jobs] == solo
    assert st["completed"] == len(jobs) and st["failed"] == 0
    with pytest.raises(capi.GpudbError):
        Server(lanes=2, heavy_lanes=2)
