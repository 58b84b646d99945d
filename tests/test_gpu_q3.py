"""Q3-like join + top-k on the GPU against the CPU oracle, bit-exact: the default and 10x
configurations, randomised predicate constants, k from 1 to 64, revenue ties broken by
order date then order key, empty sides, duplicate build keys and streamed fact tables."""
import numpy as np
import pytest

from gpudbmetalbenchmark_b200 import capi
from gpudbmetalbenchmark_b200.engine import q3_to_list

pytestmark = pytest.mark.gpu

MODES = [capi.JOIN_GLOBAL, capi.JOIN_RADIX, capi.JOIN_DIRECT]


def run(engine, cu, od, li, mode=capi.JOIN_GLOBAL, location=capi.MEM_DEVICE, **kw):
    tc, to = engine.upload("customer", cu), engine.upload("orders", od)
    tl = engine.upload("lineitem", li, location=location)
    try:
        return engine.q3(tc, to, tl, join_mode=mode, **kw)
    finally:
        for t in (tc, to, tl):
            engine.free(t)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("sizes,seed", [((150_000, 1_500_000, 6_000_000), 42), ((3000, 20000, 80000), 1),
                                        ((10, 40, 100), 2), ((1, 1, 1), 3)])
def test_q3_matches_oracle(engine, orc, mode, sizes, seed):
    cu, od, li = orc.q3_tables(*sizes, seed)
    assert run(engine, cu, od, li, mode) == orc.q3(cu, od, li)


@pytest.mark.parametrize("mode", MODES)
def test_q3_large_customer_key_range(engine, orc, mode):
    """1.7M customer keys: a customer bitmap too large for the shared-memory copy is tested in
    place by the orders filter (small ones are copied; the other tests cover those)."""
    cu, od, li = orc.q3_tables(1_700_000, 400_000, 1_600_000, 21)
    assert run(engine, cu, od, li, mode) == orc.q3(cu, od, li)


@pytest.mark.parametrize("mode", MODES)
def test_q3_random_constants_and_k(engine, orc, mode):
    rng = np.random.default_rng(5)
    cu, od, li = orc.q3_tables(20_000, 200_000, 800_000, 11)
    tc, to, tl = engine.upload("customer", cu), engine.upload("orders", od), engine.upload("lineitem", li)
    try:
        for _ in range(12):
            seg = int(rng.integers(0, 5))
            d = int(rng.integers(0, 2406))
            s = int(rng.integers(0, 2527))
            k = int(rng.choice([1, 3, 10, 33, 64]))
            got = engine.q3(tc, to, tl, segment=seg, order_date_lt=d, ship_date_gt=s, k=k, join_mode=mode)
            assert got == orc.q3(cu, od, li, seg, d, s, k), (seg, d, s, k)
    finally:
        for t in (tc, to, tl):
            engine.free(t)


def tie_tables(n_or):
    cu = dict(cust_key=np.arange(10, dtype=np.int32), segment=np.ones(10, np.uint8))
    od = dict(order_key=(4 * np.arange(n_or) + 1).astype(np.int32),
              cust_key=(np.arange(n_or) % 10).astype(np.int32),
              order_date=(np.arange(n_or) % 3).astype(np.int32))
    li = dict(order_key=od["order_key"].copy(), ship_date=np.full(n_or, 2000, np.int32),
              ext_price=np.full(n_or, 123456, np.int64), discount=np.full(n_or, 4, np.int32))
    return cu, od, li


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("n_or", [5000, 40000])
def test_q3_ties_break_by_date_then_key(engine, orc, mode, n_or):
    """All revenues equal: the global table's select pass keeps every group as a candidate
    (5000: ranked from the candidate buffer; 40000: more than the buffer holds, so the last
    block merges the whole table)."""
    cu = dict(cust_key=np.arange(10, dtype=np.int32), segment=np.ones(10, np.uint8))
    od = dict(order_key=(4 * np.arange(n_or) + 1).astype(np.int32),
              cust_key=(np.arange(n_or) % 10).astype(np.int32),
              order_date=(np.arange(n_or) % 3).astype(np.int32))
    # every order gets one row with the same revenue: the order is date asc, key asc
    li = dict(order_key=od["order_key"].copy(), ship_date=np.full(n_or, 2000, np.int32),
              ext_price=np.full(n_or, 123456, np.int64), discount=np.full(n_or, 4, np.int32))
    got = run(engine, cu, od, li, mode, k=64)
    assert got == orc.q3(cu, od, li, k=64)
    assert [r[0] for r in got[0][:3]] == [1, 13, 25]


def test_q3_near_ties_in_one_revenue_bin(engine, orc):
    """Revenues within a few units of each other share a histogram bin: the select pass
    ranks them by the full revenue, then date and key."""
    rng = np.random.default_rng(8)
    n_or = 30000
    cu, od, li = tie_tables(n_or)
    li["ext_price"] = (1_000_000 + rng.integers(0, 40, n_or)).astype(np.int64)
    for k in (1, 10, 64):
        assert run(engine, cu, od, li, k=k) == orc.q3(cu, od, li, k=k)


def test_q3_batched_ties_match_oracle(engine, orc):
    """The batched Q3 (several requests over one set of tables) runs the same select pass:
    equal and near-equal revenues give the oracle's order for every request."""
    import ctypes as C
    n_or = 20000
    cu, od, li = tie_tables(n_or)
    li["ext_price"][::3] += 1
    tc, to, tl = engine.upload("customer", cu), engine.upload("orders", od), engine.upload("lineitem", li)
    try:
        tables = capi.Q3Tables(tc.struct(), to.struct(), tl.lineitem())
        cases = [(1, 3, 1500, 64), (1, 2, 1500, 10), (1, 1, 1999, 1), (2, 3, 1500, 5)]
        reqs, outs = (capi.Request * len(cases))(), []
        for i, (seg, d, s, k) in enumerate(cases):
            reqs[i].pipeline = capi.PIPE_Q3
            reqs[i].q3 = C.pointer(tables)
            reqs[i].q3p = capi.Q3Params(seg, d, s, k, capi.JOIN_GLOBAL, 0)
            outs.append(capi.Q3Result())
            reqs[i].q3_out = C.pointer(outs[-1])
        engine._check(engine.lib.gpudb_batch_run(engine.ctx, reqs, len(cases), None, None))
        for i, (seg, d, s, k) in enumerate(cases):
            assert reqs[i].status == capi.OK
            assert q3_to_list(outs[i]) == orc.q3(cu, od, li, seg, d, s, k), cases[i]
    finally:
        for t in (tc, to, tl):
            engine.free(t)


@pytest.mark.parametrize("mode", MODES)
def test_q3_empty_sides(engine, orc, mode):
    cu, od, li = orc.q3_tables(100, 1000, 4000, 4)
    none = dict(order_key=li["order_key"][:0], ship_date=li["ship_date"][:0], ext_price=li["ext_price"][:0],
                discount=li["discount"][:0])
    assert run(engine, cu, od, none, mode) == ([], 0)
    # no qualifying customer
    assert run(engine, cu, od, li, mode, segment=9) == ([], 0)
    # no qualifying order date
    assert run(engine, cu, od, li, mode, order_date_lt=0) == ([], 0)


@pytest.mark.parametrize("mode", MODES)
def test_q3_duplicate_build_key_reported(engine, orc, mode):
    cu, od, li = orc.q3_tables(100, 1000, 4000, 4)
    od["order_key"][7] = od["order_key"][8]
    od["order_date"][7] = od["order_date"][8] = 0
    od["cust_key"][7] = od["cust_key"][8]
    cu["segment"][od["cust_key"][8]] = 1
    with pytest.raises(capi.GpudbError) as e:
        run(engine, cu, od, li, mode)
    assert e.value.code == capi.E_INVALID


def test_q3_auto_mode_picks_the_direct_map(engine, orc):
    """AUTO takes the direct map when the orders' key range fits 30% of device memory (any
    realistic range on a 180 GB B200) and reports the mode that ran; the direct mode refuses
    orders without a key bound, and a key above the declared bound is an error."""
    import ctypes as C
    cu, od, li = orc.q3_tables(2000, 20_000, 80_000, 6)
    tc, to, tl = engine.upload("customer", cu), engine.upload("orders", od), engine.upload("lineitem", li)
    try:
        r = capi.Q3Result()
        engine.q3(tc, to, tl, join_mode=capi.JOIN_AUTO, out=r, async_=True)
        engine.sync()
        assert r.join_mode == capi.JOIN_DIRECT
        assert q3_to_list(r) == orc.q3(cu, od, li)
        for mode in (capi.JOIN_GLOBAL, capi.JOIN_RADIX):
            engine.q3(tc, to, tl, join_mode=mode, out=r)
            assert r.join_mode == mode
        os_ = to.struct()
        os_.key_max = -1
        p = capi.Q3Params(1, 1170, 1170, 10, capi.JOIN_DIRECT, 0)
        rc = engine.lib.gpudb_q3_join_topk(engine.ctx, C.byref(tc.struct()), C.byref(os_), C.byref(tl.lineitem()),
                                           C.byref(p), C.byref(r), None, None)
        assert rc == capi.E_INVALID
        os_.key_max = int(od["order_key"].max()) - 4   # the largest key is above the bound
        p.order_date_lt = 2406
        p.segment = int(cu["segment"][od["cust_key"][np.argmax(od["order_key"])]])
        rc = engine.lib.gpudb_q3_join_topk(engine.ctx, C.byref(tc.struct()), C.byref(os_), C.byref(tl.lineitem()),
                                           C.byref(p), C.byref(r), None, None)
        assert rc == capi.E_KEY_RANGE
    finally:
        for t in (tc, to, tl):
            engine.free(t)


@pytest.mark.parametrize("mode", MODES)
def test_q3_streamed_fact_table(engine, orc, mode):
    cu, od, li = orc.q3_tables(5000, 50_000, 200_003, 8)
    engine.set_chunk_rows(30_000)
    try:
        assert run(engine, cu, od, li, mode, location=capi.MEM_HOST) == orc.q3(cu, od, li)
    finally:
        engine.set_chunk_rows(64 << 20)


@pytest.mark.parametrize("mode", MODES)
def test_q3_10x_configuration(engine, orc, mode):
    """Config 2 at 10x rows: 1.5M customers, 15M orders, 60M lineitem rows."""
    cu, od, li = orc.q3_tables(1_500_000, 15_000_000, 60_000_000, 42)
    assert run(engine, cu, od, li, mode) == orc.q3(cu, od, li)


@pytest.mark.parametrize("bits", [11, 12, 13])
def test_q3_radix_in_two_passes(engine, orc, bits):
    """More than 1024 partitions take two partitioning passes (the second stable, so each
    final partition stays contiguous): the result equals the oracle's."""
    cu, od, li = orc.q3_tables(3000, 20000, 80000, 5)
    assert run(engine, cu, od, li, capi.JOIN_RADIX, radix_bits=bits) == orc.q3(cu, od, li)
