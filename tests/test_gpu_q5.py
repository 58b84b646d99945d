"""Q5 (local supplier volume) on the GPU against the CPU oracle, bit-exact: SF-1 sizes, every
region, random windows, host-resident lineitem, keys past the dimension tables, empty sides
and key-range errors."""
import numpy as np
import pytest

from gpudbmetalbenchmark_b200 import capi

pytestmark = pytest.mark.gpu


def upload(engine, cu, su, od, li, location=capi.MEM_DEVICE):
    return (engine.upload("customer", cu), engine.upload("supplier", su), engine.upload("orders", od),
            engine.upload("lineitem", li, location=location))


def free(engine, *ts):
    for t in ts:
        engine.free(t)


@pytest.mark.parametrize("sizes,seed", [((150_000, 10_000, 1_500_000, 6_000_000), 42), ((3000, 200, 20000, 80000), 1),
                                        ((10, 4, 40, 100), 2)])
def test_q5_matches_oracle(engine, orc, sizes, seed):
    cu, su, od, li = orc.q5_tables(*sizes, seed)
    ts = upload(engine, cu, su, od, li)
    try:
        assert engine.q5(*ts) == orc.q5(cu, su, od, li)
    finally:
        free(engine, *ts)


def test_q5_regions_and_windows(engine, orc):
    rng = np.random.default_rng(8)
    cu, su, od, li = orc.q5_tables(20_000, 1_000, 200_000, 800_000, 12)
    ts = upload(engine, cu, su, od, li)
    try:
        for region in capi.REGION_NAMES:
            lo = int(rng.integers(0, 2000))
            hi = lo + int(rng.integers(1, 800))
            assert engine.q5(*ts, lo, hi, region) == orc.q5(cu, su, od, li, lo, hi, capi.region_mask(region)), region
    finally:
        free(engine, *ts)


def test_q5_streamed_lineitem(engine, orc):
    cu, su, od, li = orc.q5_tables(5000, 400, 50_000, 230_001, 5)
    old = engine.get_option(capi.OPT_CHUNK_ROWS)
    engine.set_option(capi.OPT_CHUNK_ROWS, 50_000)
    ts = upload(engine, cu, su, od, li, location=capi.MEM_HOST)
    try:
        assert engine.q5(*ts, 0, 2406) == orc.q5(cu, su, od, li, 0, 2406)
    finally:
        engine.set_option(capi.OPT_CHUNK_ROWS, old)
        free(engine, *ts)


def test_q5_keys_past_the_tables_and_empty_sides(engine, orc):
    cu, su, od, li = orc.q5_tables(2000, 100, 10_000, 40_000, 7)
    li = dict(li)
    sk = li["supp_key"].copy()
    sk[::9] = 5000      # no such supplier: matches nothing
    ok = li["order_key"].copy()
    ok[::13] = 10 ** 6  # no such order
    li["supp_key"], li["order_key"] = sk, ok
    ts = upload(engine, cu, su, od, li)
    try:
        assert engine.q5(*ts, 0, 2406) == orc.q5(cu, su, od, li, 0, 2406)
    finally:
        free(engine, *ts)
    empty = {k: v[:0] for k, v in su.items()}
    ts = upload(engine, cu, empty, od, li)
    try:
        assert engine.q5(*ts, 0, 2406) == []
    finally:
        free(engine, *ts)


def test_q5_key_range_error(engine, orc):
    cu, su, od, li = orc.q5_tables(200, 20, 1000, 4000, 3)
    tc = engine.upload("customer", cu, key_max={"key": 150})
    ts = (tc, engine.upload("supplier", su), engine.upload("orders", od), engine.upload("lineitem", li))
    try:
        with pytest.raises(capi.GpudbError) as e:
            engine.q5(*ts)
        assert e.value.code == capi.E_KEY_RANGE
    finally:
        free(engine, *ts)
