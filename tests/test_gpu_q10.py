"""Q10 (returned item reporting) on the GPU against the CPU oracle, bit-exact: SF-1 sizes,
random windows and k, ties in revenue (broken by customer key), host-resident lineitem,
sparse customer tables, empty sides and key-range errors."""
import numpy as np
import pytest

from gpudbmetalbenchmark_b200 import capi

pytestmark = pytest.mark.gpu


def upload(engine, cu, od, li, location=capi.MEM_DEVICE, cu_key_max=None):
    tc = engine.upload("customer", cu, key_max=None if cu_key_max is None else {"key": cu_key_max})
    return tc, engine.upload("orders", od), engine.upload("lineitem", li, location=location)


def free(engine, *ts):
    for t in ts:
        engine.free(t)


@pytest.mark.parametrize("sizes,seed", [((150_000, 1_500_000, 6_000_000), 42), ((3000, 20000, 80000), 1),
                                        ((10, 40, 100), 2), ((1, 1, 1), 3)])
def test_q10_matches_oracle(engine, orc, sizes, seed):
    cu, od, li = orc.q10_tables(*sizes, seed)
    ts = upload(engine, cu, od, li)
    try:
        assert engine.q10(*ts) == orc.q10(cu, od, li)
    finally:
        free(engine, *ts)


def test_q10_random_windows_and_k(engine, orc):
    rng = np.random.default_rng(4)
    cu, od, li = orc.q10_tables(20_000, 200_000, 800_000, 9)
    ts = upload(engine, cu, od, li)
    try:
        for _ in range(10):
            lo = int(rng.integers(0, 2400))
            hi = lo + int(rng.integers(1, 600))
            k = int(rng.choice([1, 5, 20, 64]))
            assert engine.q10(*ts, lo, hi, k) == orc.q10(cu, od, li, lo, hi, k), (lo, hi, k)
    finally:
        free(engine, *ts)


def test_q10_ties_break_by_customer_key(engine, orc):
    n = 3000
    cu = dict(cust_key=np.arange(n, dtype=np.int32))
    od = dict(order_key=(4 * np.arange(n) + 1).astype(np.int32), cust_key=(np.arange(n)[::-1] % n).astype(np.int32),
              order_date=np.full(n, 700, np.int32))
    li = dict(order_key=od["order_key"].copy(), flag=np.full(n, 2, np.uint8), ext_price=np.full(n, 5000, np.int64),
              discount=np.full(n, 3, np.int32))
    ts = upload(engine, cu, od, li)
    try:
        got = engine.q10(*ts, k=64)
        assert got == orc.q10(cu, od, li, k=64)
        assert [c for c, _ in got[0][:3]] == [0, 1, 2] and got[1] == n
    finally:
        free(engine, *ts)


def test_q10_streamed_lineitem_and_sparse_customers(engine, orc):
    cu, od, li = orc.q10_tables(5000, 50_000, 230_001, 17)
    cu2 = dict(cust_key=cu["cust_key"][::3].copy())   # two customers in three are missing
    old = engine.get_option(capi.OPT_CHUNK_ROWS)
    engine.set_option(capi.OPT_CHUNK_ROWS, 50_000)
    ts = upload(engine, cu2, od, li, location=capi.MEM_HOST, cu_key_max=4999)
    try:
        assert engine.q10(*ts, 0, 2406, 64) == orc.q10(cu2, od, li, 0, 2406, 64, cu_key_max=4999)
    finally:
        engine.set_option(capi.OPT_CHUNK_ROWS, old)
        free(engine, *ts)


def test_q10_empty_sides_and_key_range(engine, orc):
    cu, od, li = orc.q10_tables(100, 1000, 4000, 6)
    for c, o, l in ((cu, od, {k: v[:0] for k, v in li.items()}), (cu, {k: v[:0] for k, v in od.items()}, li)):
        ts = upload(engine, c, o, l)
        try:
            assert engine.q10(*ts, 0, 2406) == ([], 0)
        finally:
            free(engine, *ts)
    tc = engine.upload("customer", cu)
    to = engine.upload("orders", od, key_max={"order_key": int(od["order_key"].max()) - 8, "cust_key": 99})
    tl = engine.upload("lineitem", li)
    try:
        with pytest.raises(capi.GpudbError) as e:
            engine.q10(tc, to, tl, 0, 2406)
        assert e.value.code == capi.E_KEY_RANGE
    finally:
        free(engine, tc, to, tl)
