"""Parity of the sm_100a generator and scan kernels (Q6-like, Q1-like) against the CPU
oracle, bit-exact, through the C ABI. Edge cases follow the reference's inputs: empty and
ragged tables, unaligned column starts, all/none/one row passing, maximum values, one
group, streamed host tables with ragged chunks, and the full 60M-row configuration."""
import ctypes as C

import numpy as np
import pytest

from gpudbmetalbenchmark_b200 import capi
from gpudbmetalbenchmark_b200.engine import Q1_COLS

pytestmark = pytest.mark.gpu

GEN_CASES = [  # column id, generator kwargs
    (1, {}), (2, {}), (3, {}), (4, {}), (5, {}), (6, {}), (7, {}),
    (8, dict(n_orders=1000, order_mode=1)), (8, dict(n_orders=1000, order_mode=2)),
    (9, dict(n_parts=5000)), (10, dict(n_parts=5000, n_supp=400)),
    (20, {}), (21, {}), (30, {}), (31, dict(n_cust=777)), (32, {}), (40, {}), (41, {}), (50, {}), (51, {}),
    (60, {}), (61, dict(n_supp=400)), (62, {}),
]


@pytest.mark.parametrize("col,kw", GEN_CASES)
@pytest.mark.parametrize("n,off", [(1, 0), (4099, 0), (100_000, 12_345)])
def test_device_generator_matches_oracle(engine, orc, col, kw, n, off):
    w = engine.lib.gpudb_column_width(col)
    dptr = engine.device_array(n * w)
    spec = capi.GenSpec(seed=17, row_offset=off, n_rows=n, order_mode=kw.get("order_mode", 0),
                        n_orders=kw.get("n_orders", 0), n_cust=kw.get("n_cust", 0), n_parts=kw.get("n_parts", 0),
                        n_supp=kw.get("n_supp", 0))
    engine._check(engine.lib.gpudb_generate(engine.ctx, C.byref(spec), col, dptr, capi.MEM_DEVICE))
    got = engine.to_host(dptr, n, orc.DT[w])
    engine.device_free(dptr)
    want = orc.gen(col, n, 17, off, **kw)
    host = np.empty_like(want)
    engine._check(engine.lib.gpudb_generate(None, C.byref(spec), col, host.ctypes.data, capi.MEM_HOST))
    assert np.array_equal(got, want)
    assert np.array_equal(host, want)


def upload_li(engine, li):
    return engine.upload("lineitem", li)


@pytest.mark.parametrize("n", [0, 1, 3, 4, 5, 31, 33, 127, 129, 1000, 4097, 100_003])
def test_q6_q1_small_sizes(engine, orc, n):
    li = orc.lineitem(n, seed=n + 1)
    t = upload_li(engine, li)
    try:
        assert engine.q6(t) == orc.q6(li)
        assert engine.q6(t, 0, 2527, 0, 10, 51) == orc.q6(li, 0, 2527, 0, 10, 51)
        assert engine.q1(t) == orc.q1(li)
        assert engine.q1(t, 100) == orc.q1(li, 100)
    finally:
        engine.free(t)


@pytest.mark.parametrize("variant", [1, 2, 3, 4, 5, 6, 7, 8, 9, 10])
@pytest.mark.parametrize("n", [2047, 2048, 2049, 3 * 4096 + 5, 1_000_003])
def test_q1_every_kernel_variant(engine, orc, variant, n):
    """TMA-staged tiles (1), 128-bit loads (2) and one row per thread (3) agree exactly."""
    li = orc.lineitem(n, seed=n)
    t = upload_li(engine, li)
    try:
        engine.set_scan_variant(variant)
        assert engine.q1(t) == orc.q1(li)
        assert engine.q1(t, 700) == orc.q1(li, 700)
        assert engine.q1(t.lineitem(n_rows=n - 1, row_offset=1)) == orc.q1({k: v[1:] for k, v in li.items()})
    finally:
        engine.set_scan_variant(0)
        engine.free(t)


@pytest.mark.parametrize("off", [1, 2, 3, 5])
def test_unaligned_column_starts(engine, orc, off):
    n = 50_001
    li = orc.lineitem(n, seed=5)
    t = upload_li(engine, li)
    try:
        view = t.lineitem(n_rows=n - off, row_offset=off)
        sub = {k: v[off:] for k, v in li.items()}
        assert engine.q6(view) == orc.q6(sub)
        assert engine.q1(view) == orc.q1(sub)
    finally:
        engine.free(t)


def test_predicate_edges(engine, orc):
    n = 70_000
    li = orc.lineitem(n, seed=9)
    t = upload_li(engine, li)
    try:
        # all rows pass / none pass / exactly one row passes
        assert engine.q6(t, 0, 2527, 0, 10, 51) == orc.q6(li, 0, 2527, 0, 10, 51)
        assert engine.q6(t, 5, 5, 0, 10, 51) == (0, 0)
        r = int(np.argmax(li["ship_date"]))
        s = int(li["ship_date"][r])
        one = orc.q6(li, s, s + 1, 0, 10, 51)
        assert engine.q6(t, s, s + 1, 0, 10, 51) == one
        assert engine.q1(t, -1) == {}
        assert engine.q1(t, 2526) == orc.q1(li, 2526)
    finally:
        engine.free(t)


def test_max_values_and_single_group(engine, orc):
    n = 40_000
    li = orc.lineitem(n, seed=10)
    li["ext_price"][:] = 50 * 209900
    li["quantity"][:] = 50
    li["discount"][:] = 0
    li["tax"][:] = 8
    li["flag"][:] = 2
    li["status"][:] = 1
    t = upload_li(engine, li)
    try:
        got = engine.q1(t)
        assert list(got) == [(2, 1)]
        assert got == orc.q1(li)
    finally:
        engine.free(t)
    # the edge of the exact-arithmetic domain
    li["ext_price"][:] = (1 << 36) - 1
    li["discount"][:] = 100
    li["tax"][:] = 100
    li["quantity"][:] = 65535
    t = upload_li(engine, li)
    try:
        assert engine.q1(t) == orc.q1(li)
    finally:
        engine.free(t)


def test_domain_violation_is_reported(engine, orc):
    li = orc.lineitem(1000, seed=3)
    li["discount"][17] = 101
    li["ship_date"][17] = 0
    t = upload_li(engine, li)
    try:
        with pytest.raises(capi.GpudbError) as e:
            engine.q1(t)
        assert e.value.code == capi.E_INVALID
        # rows outside the filter do not count
        li["ship_date"][17] = 2500
        t2 = upload_li(engine, li)
        assert engine.q1(t2) == orc.q1(li)
        engine.free(t2)
    finally:
        engine.free(t)


def test_bad_arguments(engine):
    li = capi.Lineitem()
    li.n_rows = 10
    li.location = capi.MEM_DEVICE
    with pytest.raises(capi.GpudbError) as e:
        engine.q6(li)
    assert e.value.code == capi.E_INVALID
    li.location = 7
    with pytest.raises(capi.GpudbError):
        engine.q1(li)


@pytest.mark.parametrize("chunk", [16, 1000, 4096, 33_333])
def test_streamed_host_table(engine, orc, chunk):
    n = 100_003
    li = orc.lineitem(n, seed=21)
    t = engine.upload("lineitem", li, location=capi.MEM_HOST)
    try:
        engine.set_chunk_rows(chunk)
        tm = capi.Timing()
        assert engine.q6(t, timing=tm) == orc.q6(li)
        assert tm.chunks == (n + ((chunk + 15) // 16 * 16) - 1) // ((chunk + 15) // 16 * 16)
        assert tm.h2d_bytes == 20 * n
        assert engine.q1(t) == orc.q1(li)
    finally:
        engine.set_chunk_rows(64 << 20)
        engine.free(t)


def _scan_requests(li_struct, params):
    """gpudb_request array of ("q6", (lo, hi, dlo, dhi, qlt), rows) and ("q1", (ship_le,),
    rows) requests over one table (rows = (begin, end) or None), with their result structs."""
    reqs = (capi.Request * len(params))()
    outs = []
    for r, (kind, args, rows) in zip(reqs, params):
        r.li = C.pointer(li_struct)
        if kind == "q6":
            r.pipeline, r.q6 = capi.PIPE_Q6, capi.Q6Params(*args)
            o = capi.Q6Result()
            r.q6_out = C.pointer(o)
        else:
            r.pipeline, r.q1 = capi.PIPE_Q1, capi.Q1Params(args[0], 0)
            o = capi.Q1Result()
            r.q1_out = C.pointer(o)
        if rows:
            r.row_begin, r.row_end = rows
        outs.append(o)
    return reqs, outs


@pytest.mark.parametrize("chunk", [16, 1000, 33_333, 64 << 20])
def test_batched_scans_of_host_table_share_the_copy(engine, orc, chunk):
    """Q6 and Q1 requests over one host-resident table in one batch: the table crosses the
    host link once (26 B/row for the union of the columns), and every result equals the
    oracle's, bit-exactly, with ragged chunks and row ranges."""
    from gpudbmetalbenchmark_b200.engine import q1_to_dict
    n = 100_003
    li = orc.lineitem(n, seed=23)
    t = engine.upload("lineitem", li, location=capi.MEM_HOST)
    ls = t.lineitem()
    sub = lambda a, b: {k: v[a:b] for k, v in li.items()}  # noqa: E731

    def check(params, h2d=None):
        reqs, outs = _scan_requests(ls, params)
        tm = capi.Timing()
        engine._check(engine.lib.gpudb_batch_run(engine.ctx, reqs, len(params), C.byref(tm), None))
        if h2d is not None:
            assert tm.h2d_bytes == h2d
        for r, o, (kind, args, rows) in zip(reqs, outs, params):
            assert r.status == capi.OK
            part = sub(*rows) if rows else li
            if kind == "q6":
                assert (o.revenue, o.rows_matched) == orc.q6(part, *args)
            else:
                assert q1_to_dict(o) == orc.q1(part, args[0])

    try:
        engine.set_chunk_rows(chunk)
        check([("q6", (365, 730, 5, 7, 24), None), ("q1", (2436,), None), ("q6", (0, 2527, 0, 10, 51), None),
               ("q1", (1200,), None), ("q6", (100, 900, 2, 8, 30), None)], h2d=26 * n)
        # Q6 alone: only its four columns cross
        check([("q6", (365, 730, 5, 7, 24), None), ("q6", (0, 1000, 3, 9, 40), None)], h2d=20 * n)
        # row ranges: each range streams once for the requests over it
        check([("q6", (365, 730, 5, 7, 24), (1000, 60_001)), ("q1", (2436,), (7, 99_000)),
               ("q1", (2000,), (7, 99_000)), ("q6", (0, 2527, 0, 10, 51), (7, 99_000))],
              h2d=20 * 59_001 + 26 * 98_993)
    finally:
        engine.set_chunk_rows(64 << 20)
        engine.free(t)


def test_async_calls_complete_at_sync(engine, orc):
    n = 200_000
    li = orc.lineitem(n, seed=4)
    t = upload_li(engine, li)
    try:
        before = engine.launches()
        outs6 = [capi.Q6Result() for _ in range(40)]
        outs1 = [capi.Q1Result() for _ in range(40)]
        tms = [capi.Timing() for _ in range(40)]
        for i in range(40):
            engine.q6(t, ship_lo=i * 50, ship_hi=i * 50 + 400, async_=True, out=outs6[i], timing=tms[i])
            engine.q1(t, ship_le=i * 60, async_=True, out=outs1[i])
        engine.sync()
        assert engine.launches() - before >= 80
        from gpudbmetalbenchmark_b200.engine import q1_to_dict
        for i in range(40):
            assert (outs6[i].revenue, outs6[i].rows_matched) == orc.q6(li, i * 50, i * 50 + 400)
            assert q1_to_dict(outs1[i]) == orc.q1(li, i * 60)
            assert tms[i].kernels == 1 and tms[i].gpu_ms > 0
    finally:
        engine.free(t)


def test_direct_results_over_reused_slots(engine, orc):
    """Device-resident Q6/Q1 calls write their result straight into the pinned host slot from
    the kernel's last block (no slot clear, no copy back). Over more async calls than there
    are result slots (1024), every result must equal the oracle's, whatever an earlier call
    left in the slot, and a call whose Q1 status reports a domain error must not leak that
    status into the calls after it. The same calls on a host-resident table (streamed, with
    the slot cleared and copied back) give the same words."""
    from gpudbmetalbenchmark_b200.engine import q1_to_dict
    n = 50_001
    li = orc.lineitem(n, seed=44)
    bad = {k: v.copy() for k, v in li.items()}
    bad["discount"][7] = 101
    bad["ship_date"][7] = 0
    t, tb = upload_li(engine, li), upload_li(engine, bad)
    th = engine.upload("lineitem", li, location=capi.MEM_HOST)
    try:
        q6p = [(i * 90, i * 90 + 500, i % 6, i % 6 + 4, 20 + i) for i in range(12)]
        q1p = [i * 230 for i in range(12)]
        want6 = [orc.q6(li, *p) for p in q6p]
        want1 = [orc.q1(li, s) for s in q1p]
        calls = 1100
        o6 = [capi.Q6Result() for _ in range(calls)]
        o1 = [capi.Q1Result() for _ in range(calls)]
        failed = capi.Q1Result()
        for i in range(calls):
            engine.q6(t, *q6p[i % 12], async_=True, out=o6[i])
            engine.q1(t, q1p[i % 12], async_=True, out=o1[i])
            if i == calls - 20:   # after the last drain that a full set of slots forces
                engine.q1(tb, async_=True, out=failed)
        with pytest.raises(capi.GpudbError) as e:
            engine.sync()
        assert e.value.code == capi.E_INVALID
        for i in range(calls):
            assert (o6[i].revenue, o6[i].rows_matched) == want6[i % 12]
            assert q1_to_dict(o1[i]) == want1[i % 12]
        # synchronous calls: direct (device table) and copied back (host table) agree
        for p, s in zip(q6p[:3], q1p[:3]):
            tm_d, tm_h = capi.Timing(), capi.Timing()
            assert engine.q6(t, *p, timing=tm_d) == engine.q6(th, *p, timing=tm_h) == orc.q6(li, *p)
            assert tm_d.d2h_bytes == tm_h.d2h_bytes
            r_d, r_h = capi.Q1Result(), capi.Q1Result()
            engine.q1(t, s, out=r_d)
            engine.q1(th, s, out=r_h)
            assert bytes(r_d) == bytes(r_h)
    finally:
        engine.free(t)
        engine.free(tb)
        engine.free(th)


def test_full_size_60m_bit_exact(engine, orc):
    """Config 1 at its full size: 60M rows generated on the device, both scans bit-exact
    against the oracle run on the same rows generated on the host."""
    n = 60_000_000
    t = engine.generate("lineitem", n, seed=42, columns=Q1_COLS)
    try:
        li = orc.lineitem(n, seed=42)
        assert engine.q6(t) == orc.q6(li, threads=8)
        want = orc.q1(li, threads=8)
        for variant in (1, 2, 3, 4, 5, 6, 7, 8):
            engine.set_scan_variant(variant)
            assert engine.q1(t) == want
        engine.set_scan_variant(0)
        # linearity: the two halves add up to the whole
        h = n // 2 + 3
        a = engine.q6(t.lineitem(n_rows=h))
        b = engine.q6(t.lineitem(n_rows=n - h, row_offset=h))
        assert (a[0] + b[0], a[1] + b[1]) == engine.q6(t)
    finally:
        engine.free(t)
