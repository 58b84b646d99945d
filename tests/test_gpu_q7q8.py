"""Q7 (volume shipping) and Q8 (national market share) on the GPU against the CPU oracle,
bit-exact: SF-1 sizes, other nation pairs, regions, part types and multi-year windows,
host-resident lineitem, keys past the tables, empty sides and the parameter checks."""
import numpy as np
import pytest

from gpudbmetalbenchmark_b200 import capi

pytestmark = pytest.mark.gpu
ASIA = capi.region_mask("ASIA")


def upload(engine, cu, su, pa, od, li, location=capi.MEM_DEVICE):
    return (engine.upload("customer", cu), engine.upload("supplier", su), engine.upload("part", pa),
            engine.upload("orders", od), engine.upload("lineitem", li, location=location))


def free(engine, ts):
    for t in ts:
        engine.free(t)


@pytest.mark.parametrize("sizes,seed", [((150_000, 10_000, 200_000, 1_500_000, 6_000_000), 42),
                                        ((3000, 200, 2000, 20000, 80000), 1), ((10, 4, 8, 40, 100), 2)])
def test_q7_q8_match_oracle(engine, orc, sizes, seed):
    tabs = orc.q8_tables(*sizes, seed)
    cu, su, pa, od, li = tabs
    ts = upload(engine, *tabs)
    try:
        assert engine.q7(ts[0], ts[1], ts[3], ts[4]) == orc.q7(cu, su, od, li)
        assert engine.q8(*ts) == orc.q8(*tabs)
    finally:
        free(engine, ts)


def test_q7_q8_other_parameters(engine, orc):
    rng = np.random.default_rng(3)
    tabs = orc.q8_tables(20_000, 1_000, 3_000, 200_000, 800_000, 14)
    cu, su, pa, od, li = tabs
    ts = upload(engine, *tabs)
    try:
        for _ in range(6):
            a, b = (int(x) for x in rng.integers(0, 25, 2))
            lo = int(rng.integers(-50, 2000))
            hi = lo + int(rng.integers(0, 7 * 365))
            assert engine.q7(ts[0], ts[1], ts[3], ts[4], a, b, lo, hi) == orc.q7(cu, su, od, li, a, b, lo, hi), (a, b)
            n, t = int(rng.integers(0, 25)), int(rng.integers(0, 150))
            region = capi.REGION_NAMES[int(rng.integers(0, 5))]
            got = engine.q8(*ts, n, region, t, lo, hi)
            assert got == orc.q8(*tabs, n, capi.region_mask(region), t, lo, hi), (n, region, t)
    finally:
        free(engine, ts)


def test_q7_q8_streamed_lineitem(engine, orc):
    tabs = orc.q8_tables(5000, 400, 600, 50_000, 230_001, 6)
    cu, su, pa, od, li = tabs
    old = engine.get_option(capi.OPT_CHUNK_ROWS)
    engine.set_option(capi.OPT_CHUNK_ROWS, 50_000)
    ts = upload(engine, *tabs, location=capi.MEM_HOST)
    try:
        assert engine.q7(ts[0], ts[1], ts[3], ts[4], 12, 18, 0, 2406) == orc.q7(cu, su, od, li, 12, 18, 0, 2406)
        assert engine.q8(*ts, 12, "ASIA", 7, 366, 2191) == orc.q8(*tabs, 12, ASIA, 7, 366, 2191)
    finally:
        engine.set_option(capi.OPT_CHUNK_ROWS, old)
        free(engine, ts)


def test_q7_q8_keys_past_the_tables(engine, orc):
    tabs = orc.q8_tables(2000, 100, 300, 10_000, 40_000, 7)
    cu, su, pa, od, li = tabs
    li = dict(li)
    for col, bad in (("supp_key", 5000), ("part_key", 9000), ("order_key", 10 ** 6)):
        v = li[col].copy()
        v[::7] = bad
        v[3::11] = -2
        li[col] = v
    tabs = (cu, su, pa, od, li)
    ts = upload(engine, *tabs)
    try:
        assert engine.q7(ts[0], ts[1], ts[3], ts[4], 6, 7, 0, 2406) == orc.q7(cu, su, od, li, 6, 7, 0, 2406)
        assert engine.q8(*ts, 2, "AMERICA", 40, 0, 2406) == orc.q8(*tabs, 2, capi.region_mask("AMERICA"), 40, 0, 2406)
    finally:
        free(engine, ts)


def test_q7_q8_empty_sides_and_checks(engine, orc):
    tabs = orc.q8_tables(300, 40, 100, 2000, 8000, 3)
    cu, su, pa, od, li = tabs
    empty_pa = {k: v[:0] for k, v in pa.items()}
    ts = upload(engine, cu, su, empty_pa, od, li)
    try:
        assert engine.q8(*ts) == [(1995, 0, 0), (1996, 0, 0)]
        with pytest.raises(capi.GpudbError) as e:            # more than 8 calendar years
            engine.q7(ts[0], ts[1], ts[3], ts[4], 6, 7, 0, 9 * 366)
        assert e.value.code == capi.E_INVALID
        with pytest.raises(capi.GpudbError) as e:
            engine.q8(*ts, 2, "AMERICA", 150)
        assert e.value.code == capi.E_INVALID
    finally:
        free(engine, ts)
    tc = engine.upload("customer", cu, key_max={"key": 100})   # keys above the declared bound
    ts = (tc, engine.upload("supplier", su), engine.upload("orders", od), engine.upload("lineitem", li))
    try:
        with pytest.raises(capi.GpudbError) as e:
            engine.q7(*ts)
        assert e.value.code == capi.E_KEY_RANGE
    finally:
        free(engine, ts)
