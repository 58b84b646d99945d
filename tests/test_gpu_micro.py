"""Microbenchmark operators and the radix partitioner on the GPU against the CPU oracle:
selection (bitmask + ordered row ids), exact column sum, hash-join match count (global and
radix), stable radix partitioning (identical to the oracle's, whose partition numbers are
pinned to the reference's own sf100_radix_* kernels), and all-pairs radix join."""
import numpy as np
import pytest

from gpudbmetalbenchmark_b200 import capi

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [0, 1, 31, 32, 33, 4095, 4097, 1_000_003])
@pytest.mark.parametrize("value", [0, 1000, 2527, 5000])
def test_select_lt(engine, orc, n, value):
    col = orc.gen(1, n, seed=n + 7)
    dcol = engine.to_device(col) if n else None
    bits = engine.device_array(((n + 31) // 32) * 4 + 4)
    rows = engine.device_array(n * 4 + 4)
    try:
        c = engine.select_lt(dcol, n, value, bits, rows)
        wc, wbits, wrows = orc.select_lt(col, value)
        assert c == wc
        assert np.array_equal(engine.to_host(bits, (n + 31) // 32, np.uint32), wbits)
        assert np.array_equal(engine.to_host(rows, c, np.uint32), wrows)
        assert engine.select_lt(dcol, n, value) == wc   # count only
        # bitmask only (one kernel, no per-tile counts): every word written, on a buffer of ones
        words = (n + 31) // 32
        ones = engine.to_device(np.full(words + 1, 0xFFFFFFFF, np.uint32))
        try:
            assert engine.select_lt(dcol, n, value, ones) == wc
            assert np.array_equal(engine.to_host(ones, words, np.uint32), wbits)
            if n > 1:   # the column 4 bytes past a 16-byte boundary
                wc1, wbits1, _ = orc.select_lt(col[1:], value)
                assert engine.select_lt(dcol + 4, n - 1, value, ones) == wc1
                assert np.array_equal(engine.to_host(ones, (n + 30) // 32, np.uint32), wbits1)
        finally:
            engine.device_free(ones)
    finally:
        for p in (dcol, bits, rows):
            if p:
                engine.device_free(p)


@pytest.mark.parametrize("n,off", [(0, 0), (1, 0), (5, 1), (1_000_001, 0), (1_000_001, 3), (60_000_000, 0)])
def test_sum_i32(engine, orc, n, off):
    col = orc.gen(2, n + off, seed=3)
    d = engine.to_device(col) if n + off else None
    try:
        got = engine.sum_i32(d + 4 * off if d else None, n)
        assert got == orc.sum_i32(col[off:])
    finally:
        if d:
            engine.device_free(d)


def test_sum_i32_extreme_values(engine, orc):
    col = np.full(3_000_001, np.iinfo(np.int32).max, np.int32)
    col[::2] = np.iinfo(np.int32).min
    d = engine.to_device(col)
    try:
        assert engine.sum_i32(d, len(col)) == int(col.astype(np.int64).sum())
    finally:
        engine.device_free(d)


@pytest.mark.parametrize("mode", [capi.JOIN_GLOBAL, capi.JOIN_RADIX, capi.JOIN_DIRECT])
@pytest.mark.parametrize("nb,np_,orders", [(1_500_000, 6_000_000, 1_500_000), (1000, 5000, 700), (1, 1, 1),
                                           (0, 100, 10), (100, 0, 10), (200_000, 300_000, 50_000)])
def test_hash_join_count(engine, orc, mode, nb, np_, orders):
    b = orc.gen(30, nb, seed=1) if orders >= nb else orc.gen(8, nb, seed=1, n_orders=orders, order_mode=2)
    p = orc.gen(8, np_, seed=2, n_orders=max(orders, 1) * 2, order_mode=2)
    db = engine.to_device(b) if nb else None
    dp = engine.to_device(p) if np_ else None
    try:
        assert engine.hash_join_count(db, nb, dp, np_, mode) == orc.join_count(b, p)
    finally:
        for x in (db, dp):
            if x:
                engine.device_free(x)


@pytest.mark.parametrize("bits", [0, 1, 3, 8, 9, 10, 12, 16])
@pytest.mark.parametrize("n", [1, 4096, 4097, 300_001])
def test_radix_partition_is_the_oracle_partition(engine, orc, bits, n):
    keys = orc.gen(8, n, seed=bits + 5, n_orders=max(n // 3, 1), order_mode=2)
    pay = np.arange(n, dtype=np.int32) * 7 + 3
    dk, dp = engine.to_device(keys), engine.to_device(pay)
    ko, po, off = (engine.device_array(n * 4), engine.device_array(n * 4), engine.device_array(((1 << bits) + 1) * 4))
    try:
        engine.radix_partition(dk, dp, n, bits, ko, po, off)
        wk, wp, woff = orc.radix_partition(keys, pay, bits)
        assert np.array_equal(engine.to_host(off, (1 << bits) + 1, np.uint32), woff)
        assert np.array_equal(engine.to_host(ko, n, np.int32), wk)
        assert np.array_equal(engine.to_host(po, n, np.int32), wp)
        engine.radix_partition(dk, None, n, bits, ko, po, off)   # payload = row ids
        _, rows, _ = orc.radix_partition(keys, np.arange(n, dtype=np.int32), bits)
        assert np.array_equal(engine.to_host(po, n, np.int32), rows)
    finally:
        for x in (dk, dp, ko, po, off):
            engine.device_free(x)


@pytest.mark.parametrize("bits,n", [(10, 3_000_017), (13, 2_500_001), (7, 1_300_000)])
def test_radix_partition_large_inputs(engine, orc, bits, n):
    """Inputs of many 8192-row sub-tiles per super-tile: the per-digit cursors carry the
    rows of one super-tile across its sub-tiles in input order."""
    keys = orc.gen(8, n, seed=bits, n_orders=n // 2, order_mode=1)
    pay = np.arange(n, dtype=np.int32) ^ 0x5A5A
    dk, dp = engine.to_device(keys), engine.to_device(pay)
    ko, po, off = (engine.device_array(n * 4), engine.device_array(n * 4), engine.device_array(((1 << bits) + 1) * 4))
    try:
        engine.radix_partition(dk, dp, n, bits, ko, po, off)
        wk, wp, woff = orc.radix_partition(keys, pay, bits)
        assert np.array_equal(engine.to_host(off, (1 << bits) + 1, np.uint32), woff)
        assert np.array_equal(engine.to_host(ko, n, np.int32), wk)
        assert np.array_equal(engine.to_host(po, n, np.int32), wp)
    finally:
        for x in (dk, dp, ko, po, off):
            engine.device_free(x)


@pytest.mark.parametrize("shape", [1, 2, 3, 4, 5, 6, 7])
def test_radix_partition_every_block_shape(engine, orc, shape):
    """Every scatter block shape (GPUDB_OPT_RADIX_SHAPE) gives the oracle's stable partition,
    in one pass (10 bits) and in two (13 bits), and the same join count; columns that start
    off a 16-byte boundary (which the bulk-copy ring cannot stage) give it too."""
    n = 2_000_003
    keys = orc.gen(8, n, seed=shape, n_orders=n // 3, order_mode=1)
    pay = np.arange(n, dtype=np.int32) * 3
    dk, dp = engine.to_device(keys), engine.to_device(pay)
    ko, po, off = engine.device_array(n * 4), engine.device_array(n * 4), engine.device_array(((1 << 13) + 1) * 4)
    try:
        engine.set_option(capi.OPT_RADIX_SHAPE, shape)
        for bits in (10, 13):
            engine.radix_partition(dk, dp, n, bits, ko, po, off)
            wk, wp, woff = orc.radix_partition(keys, pay, bits)
            assert np.array_equal(engine.to_host(off, (1 << bits) + 1, np.uint32), woff)
            assert np.array_equal(engine.to_host(ko, n, np.int32), wk)
            assert np.array_equal(engine.to_host(po, n, np.int32), wp)
        # one row in: both columns 4 bytes past a 16-byte boundary
        m = n - 1
        engine.radix_partition(dk + 4, dp + 4, m, 10, ko, po, off)
        wk, wp, woff = orc.radix_partition(keys[1:], pay[1:], 10)
        assert np.array_equal(engine.to_host(off, (1 << 10) + 1, np.uint32), woff)
        assert np.array_equal(engine.to_host(ko, m, np.int32), wk)
        assert np.array_equal(engine.to_host(po, m, np.int32), wp)
        b = keys[: n // 4]
        assert engine.hash_join_count(dk, n // 4, dk, n, capi.JOIN_RADIX) == orc.join_count(b, keys)
    finally:
        engine.set_option(capi.OPT_RADIX_SHAPE, 0)
        for x in (dk, dp, ko, po, off):
            engine.device_free(x)


@pytest.mark.parametrize("shape", [5, 3])
def test_radix_join_count_through_the_ring(engine, orc, shape):
    """Tables large enough that every scatter block walks several sub-tiles through its
    bulk-copy ring: the join count over 10-bit partitions (unstable, keys only) equals the
    oracle's, also for a probe side whose length is not a whole number of sub-tiles and
    starts off a 16-byte boundary (direct loads, no ring)."""
    nb, npr = 3_000_001, 12_000_017
    b = orc.gen(8, nb, seed=41, n_orders=nb // 2, order_mode=2)
    p = orc.gen(8, npr, seed=42, n_orders=nb // 2, order_mode=1)
    db, dp = engine.to_device(b), engine.to_device(p)
    try:
        engine.set_option(capi.OPT_RADIX_SHAPE, shape)
        assert engine.hash_join_count(db, nb, dp, npr, capi.JOIN_RADIX) == orc.join_count(b, p)
        assert engine.hash_join_count(db, nb, dp + 4, npr - 1, capi.JOIN_RADIX) == orc.join_count(b, p[1:])
    finally:
        engine.set_option(capi.OPT_RADIX_SHAPE, 0)
        engine.device_free(db)
        engine.device_free(dp)


def test_join_count_direct_edges(engine, orc):
    """Direct mode: a bitmap over the build keys' span [min, max]. Negative keys, the int32
    extremes among the probe keys (outside the span: no match, whatever their distance), a
    probe column off a 16-byte boundary, a span of one key, and a span of 2^30 keys or more
    (refused with GPUDB_E_KEY_RANGE, the context still usable)."""
    rng = np.random.default_rng(9)
    b = rng.integers(-500_000, 2_000_000, 300_000, dtype=np.int64).astype(np.int32)
    p = np.concatenate([rng.integers(-800_000, 2_500_000, 1_000_003, dtype=np.int64).astype(np.int32),
                        np.array([-2**31, 2**31 - 1, -500_001, 2_000_000, b.min(), b.max()], np.int32)])
    db, dp = engine.to_device(b), engine.to_device(p)
    try:
        assert engine.hash_join_count(db, len(b), dp, len(p), capi.JOIN_DIRECT) == orc.join_count(b, p)
        assert engine.hash_join_count(db, len(b), dp + 4, len(p) - 1, capi.JOIN_DIRECT) == orc.join_count(b, p[1:])
        assert engine.hash_join_count(db, 1, dp, len(p), capi.JOIN_DIRECT) == orc.join_count(b[:1], p)
    finally:
        engine.device_free(db)
        engine.device_free(dp)
    wide = np.array([5, 5 + 2**30, 17], np.int32)
    dw, dq = engine.to_device(wide), engine.to_device(np.array([5, 17, 6], np.int32))
    try:
        with pytest.raises(capi.GpudbError) as e:
            engine.hash_join_count(dw, 3, dq, 3, capi.JOIN_DIRECT)
        assert e.value.code == capi.E_KEY_RANGE
        assert engine.hash_join_count(dw, 3, dq, 3, capi.JOIN_GLOBAL) == 2
        narrow = np.array([5, 4 + 2**30, 17], np.int32)   # a span of exactly 2^30 keys is refused, 2^30 - 1 is not
        dn = engine.to_device(narrow)
        try:
            assert engine.hash_join_count(dn, 3, dq, 3, capi.JOIN_DIRECT) == 2
        finally:
            engine.device_free(dn)
    finally:
        engine.device_free(dw)
        engine.device_free(dq)


def test_radix_partition_bad_bits(engine):
    with pytest.raises(capi.GpudbError) as e:
        engine.radix_partition(None, None, 0, 17, 1, 1, 1)
    assert e.value.code == capi.E_INVALID


@pytest.mark.parametrize("nb,np_,orders", [(15_000, 60_000, 20_000), (3000, 9000, 4000), (1, 5, 1)])
def test_radix_join_pairs(engine, orc, nb, np_, orders):
    b = orc.gen(8, nb, seed=2, n_orders=orders, order_mode=2)   # duplicates on both sides
    p = orc.gen(8, np_, seed=3, n_orders=orders, order_mode=2)
    _, _, total = orc.join_pairs(b, p, 0)
    db, dp = engine.to_device(b), engine.to_device(p)
    ob, op = engine.device_array(total * 4 + 4), engine.device_array(total * 4 + 4)
    try:
        n = engine.radix_join_pairs(db, nb, dp, np_, ob, op, total)
        assert n == total
        got = sorted(zip(engine.to_host(op, n, np.int32).tolist(), engine.to_host(ob, n, np.int32).tolist()))
        wb, wp, _ = orc.join_pairs(b, p, total)
        assert got == sorted(zip(wp.tolist(), wb.tolist()))
        # a short output buffer: the total is still reported, nothing is written past it
        assert engine.radix_join_pairs(db, nb, dp, np_, ob, op, total // 2) == total
    finally:
        for x in (db, dp, ob, op):
            engine.device_free(x)


def test_radix_join_skewed_partition(engine, orc):
    """One key repeated 5000 times on the build side: its partition needs several chunks."""
    b = np.concatenate([np.full(5000, 77, np.int32), np.arange(1000, 3000, dtype=np.int32)])
    p = np.concatenate([np.full(3, 77, np.int32), np.arange(0, 4000, 7, dtype=np.int32)])
    db, dp = engine.to_device(b), engine.to_device(p)
    _, _, total = orc.join_pairs(b, p, 0)
    ob, op = engine.device_array(total * 4), engine.device_array(total * 4)
    try:
        assert engine.radix_join_pairs(db, len(b), dp, len(p), ob, op, total) == total
        got = sorted(zip(engine.to_host(op, total, np.int32).tolist(), engine.to_host(ob, total, np.int32).tolist()))
        wb, wp, _ = orc.join_pairs(b, p, total)
        assert got == sorted(zip(wp.tolist(), wb.tolist()))
        assert engine.hash_join_count(db, len(b), dp, len(p), capi.JOIN_RADIX) == orc.join_count(b, p)
    finally:
        for x in (db, dp, ob, op):
            engine.device_free(x)


def test_radix_join_count_multi_chunk_partition(engine, orc):
    """A build partition larger than one shared-memory chunk of the count kernel (one key
    40,000 times next to 20,000 distinct keys): matches are flagged per chunk and counted once."""
    b = np.concatenate([np.full(40_000, 77, np.int32), np.arange(100_000, 120_000, dtype=np.int32)])
    p = np.concatenate([np.full(5, 77, np.int32), np.arange(90_000, 130_000, 3, dtype=np.int32), np.array([76, 78], np.int32)])
    db, dp = engine.to_device(b), engine.to_device(p)
    try:
        assert engine.hash_join_count(db, len(b), dp, len(p), capi.JOIN_RADIX) == orc.join_count(b, p)
    finally:
        for x in (db, dp):
            engine.device_free(x)


def test_radix_join_pairs_in_two_passes(engine, orc):
    """2.1M build rows need 11 partition bits (two passes): every pair is found once."""
    rng = np.random.default_rng(41)
    b = (rng.permutation(2_100_000) * 3).astype(np.int32)
    p = rng.integers(0, 7_000_000, 2_500_000).astype(np.int32)
    want = np.sort(p[(p % 3 == 0) & (p < 6_300_000)])
    db, dp = engine.to_device(b), engine.to_device(p)
    ob, op = engine.device_array(len(want) * 4 + 4), engine.device_array(len(want) * 4 + 4)
    try:
        n = engine.radix_join_pairs(db, len(b), dp, len(p), ob, op, len(want))
        assert n == len(want)
        bk = b[engine.to_host(ob, n, np.int32)]
        pk = p[engine.to_host(op, n, np.int32)]
        assert np.array_equal(bk, pk)                 # each pair joins equal keys
        assert np.array_equal(np.sort(pk), want)      # and every matching probe row once
    finally:
        for x in (db, dp, ob, op):
            engine.device_free(x)


def test_radix_join_count_in_two_passes(engine):
    """16M distinct build keys need 11 partition bits in the count (two passes)."""
    b = (np.arange(16_000_000, dtype=np.int64) * 2).astype(np.int32)
    p = np.random.default_rng(43).integers(0, 40_000_000, 20_000_000).astype(np.int32)
    want = int(((p % 2 == 0) & (p < 32_000_000)).sum())
    db, dp = engine.to_device(b), engine.to_device(p)
    try:
        assert engine.hash_join_count(db, len(b), dp, len(p), capi.JOIN_RADIX) == want
    finally:
        for x in (db, dp):
            engine.device_free(x)
