"""Q4 (order priority checking) and Q12 (shipping modes and order priority) on the GPU
against the CPU oracle, bit-exact: SF-1-sized tables, clustered and scattered order keys,
randomised windows / modes / priority cuts, host-resident lineitem streamed in chunks, empty
sides, lineitem keys past the orders' key range, and order keys outside the declared range."""
import numpy as np
import pytest

from gpudbmetalbenchmark_b200 import capi

pytestmark = pytest.mark.gpu


def upload(engine, od, li, location=capi.MEM_DEVICE, od_key_max=None):
    to = engine.upload("orders", od, key_max=None if od_key_max is None else {"order_key": od_key_max})
    tl = engine.upload("lineitem", li, location=location)
    return to, tl


def free(engine, *ts):
    for t in ts:
        engine.free(t)


@pytest.mark.parametrize("n_or,n_li,seed,mode", [(1_500_000, 6_000_000, 42, 1), (200_000, 800_000, 7, 2),
                                                 (100, 300, 3, 1), (1, 1, 4, 1)])
def test_q4_q12_match_oracle(engine, orc, n_or, n_li, seed, mode):
    od, li = orc.q4_tables(n_or, n_li, seed, order_mode=mode)
    to, tl = upload(engine, od, li)
    try:
        assert engine.q4(to, tl) == orc.q4(od, li)
        assert engine.q12(to, tl) == orc.q12(od, li)
    finally:
        free(engine, to, tl)


def test_q4_q12_random_parameters(engine, orc):
    rng = np.random.default_rng(12)
    od, li = orc.q4_tables(300_000, 1_200_000, 19)
    to, tl = upload(engine, od, li)
    try:
        for _ in range(10):
            lo = int(rng.integers(-100, 2500))
            hi = lo + int(rng.integers(0, 900))
            assert engine.q4(to, tl, lo, hi) == orc.q4(od, li, lo, hi), (lo, hi)
            modes = tuple(int(x) for x in rng.integers(0, 7, 2))
            high_max = int(rng.integers(0, 6))
            got = engine.q12(to, tl, lo, hi, modes, high_max)
            assert got == orc.q12(od, li, lo, hi, modes, high_max), (lo, hi, modes, high_max)
    finally:
        free(engine, to, tl)


def test_q4_q12_streamed_lineitem(engine, orc):
    """Host-resident lineitem goes through the chunk ring (50,000-row chunks here)."""
    od, li = orc.q4_tables(60_000, 230_001, 23)
    to, tl = upload(engine, od, li, location=capi.MEM_HOST)
    old = engine.get_option(capi.OPT_CHUNK_ROWS)
    engine.set_option(capi.OPT_CHUNK_ROWS, 50_000)
    try:
        t = capi.Timing()
        assert engine.q4(to, tl, timing=t) == orc.q4(od, li)
        assert t.chunks == 5 and t.h2d_bytes == 230_001 * 12
        assert engine.q12(to, tl, 0, 2600) == orc.q12(od, li, 0, 2600)
    finally:
        engine.set_option(capi.OPT_CHUNK_ROWS, old)
        free(engine, to, tl)


def test_q4_q12_empty_sides(engine, orc):
    od, li = orc.q4_tables(1000, 4000, 2)
    empty_li = {k: v[:0] for k, v in li.items()}
    empty_od = {k: v[:0] for k, v in od.items()}
    to, tl = upload(engine, od, empty_li)
    try:
        assert engine.q4(to, tl, 0, 3000) == [0] * 5
        assert engine.q12(to, tl, 0, 3000) == [(0, 0), (0, 0)]
    finally:
        free(engine, to, tl)
    to, tl = upload(engine, empty_od, li)
    try:
        assert engine.q4(to, tl, 0, 3000) == [0] * 5
        # no orders: every qualifying row is low
        assert engine.q12(to, tl, 0, 3000) == orc.q12(empty_od, li, 0, 3000, or_key_max=-1)
    finally:
        free(engine, to, tl)


def test_lineitem_keys_past_the_orders(engine, orc):
    """Lineitem rows whose order key is beyond the orders' key range (or negative) match no
    order: Q4 ignores them, Q12 counts them low."""
    od, li = orc.q4_tables(5000, 20000, 31)
    li = dict(li)
    k = li["order_key"].copy()
    k[::7] = 4 * 5000 + 77
    k[3::11] = -5
    li["order_key"] = k
    to, tl = upload(engine, od, li)
    try:
        assert engine.q4(to, tl, 0, 2406) == orc.q4(od, li, 0, 2406)
        assert engine.q12(to, tl, 0, 2600) == orc.q12(od, li, 0, 2600)
    finally:
        free(engine, to, tl)


def test_order_key_outside_declared_range(engine, orc):
    """An order key above the declared key_max is reported (E_KEY_RANGE), not dropped."""
    od, li = orc.q4_tables(2000, 8000, 5)
    to, tl = upload(engine, od, li, od_key_max=int(od["order_key"].max()) - 10)
    try:
        with pytest.raises(capi.GpudbError) as e:
            engine.q4(to, tl, 0, 2406)
        assert e.value.code == capi.E_KEY_RANGE
        with pytest.raises(capi.GpudbError) as e:
            engine.q12(to, tl)
        assert e.value.code == capi.E_KEY_RANGE
    finally:
        free(engine, to, tl)


def test_missing_columns_are_rejected(engine, orc):
    od, li = orc.q4_tables(100, 400, 5)
    to, tl = upload(engine, {k: v for k, v in od.items() if k != "priority"}, li)
    try:
        with pytest.raises(capi.GpudbError) as e:
            engine.q4(to, tl)
        assert e.value.code == capi.E_INVALID
    finally:
        free(engine, to, tl)
