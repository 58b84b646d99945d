"""Q13 (customer distribution) on the GPU against the CPU oracle, bit-exact: SF-1 sizes,
other word pairs, hand-written comments at the pattern's edge cases (adjacent words, words
in the wrong order, a word cut by the 80-byte slot end, one-letter words, empty comments),
customers without orders, orders of unknown customers, and the count and word limits."""
import numpy as np
import pytest

from gpudbmetalbenchmark_b200 import capi

pytestmark = pytest.mark.gpu


def run(engine, cu, od, *words, cu_key_max=None):
    tc = engine.upload("customer", cu, key_max=None if cu_key_max is None else {"key": cu_key_max})
    to = engine.upload("orders", od)
    try:
        return engine.q13(tc, to, *words)
    finally:
        engine.free(tc)
        engine.free(to)


@pytest.mark.parametrize("n_cu,n_or,seed", [(150_000, 1_500_000, 42), (20_000, 90_000, 3), (1, 1, 5), (7, 0, 6)])
def test_q13_matches_oracle(engine, orc, n_cu, n_or, seed):
    cu, od = orc.q13_tables(n_cu, max(n_or, 1), seed)
    if n_or == 0:
        od = {k: v[:0] for k, v in od.items()}
    assert run(engine, cu, od) == orc.q13(cu, od)


@pytest.mark.parametrize("w1,w2", [(b"pinto", b"beans"), (b"s", b"s"), (b"even", b"bold"), (b"y", b"e"),
                                   (b"instructions", b"instructions")])
def test_q13_other_words(engine, orc, w1, w2):
    cu, od = orc.q13_tables(3000, 40_000, 11)
    assert run(engine, cu, od, w1, w2) == orc.q13(cu, od, w1, w2)


def test_q13_hand_written_comments(engine, orc):
    texts = [b"special requests", b"requests special", b"specialrequests", b"xspecialx yrequestsy",
             b"special", b"requests", b"", b"spe cial requests", b"special reque sts",
             b"a" * 72 + b"special",                      # word 1 ends at the slot's last text byte
             b"special " + b"b" * 63 + b"requests",        # 79 characters, word 2 at the very end
             b"special " + b"b" * 64 + b"request",         # word 2 cut off
             b"sspecial rrequests", b"special special requests requests"]
    n = len(texts)
    od = dict(cust_key=np.arange(n, dtype=np.int32) % 4, comment=np.array(texts, dtype="S80"))
    cu = dict(cust_key=np.arange(6, dtype=np.int32))   # customers 4 and 5 have no orders
    got = run(engine, cu, od)
    assert got == orc.q13(cu, od)
    # direct count: the comments that are NOT LIKE '%special%requests%'
    keep = [t for t in texts if not (b"special" in t and b"requests" in t.split(b"special", 1)[1])]
    assert sum(c * d for c, d in got) == len(keep)


def test_q13_orders_of_unknown_customers(engine, orc):
    cu, od = orc.q13_tables(500, 20_000, 13)
    od = dict(od)
    ck = od["cust_key"].copy()
    ck[::5] = 900      # beyond the customers' key range: counted for nobody
    ck[1::9] = -3
    od["cust_key"] = ck
    assert run(engine, cu, od) == orc.q13(cu, od)
    # sparse customer keys: only the listed customers are in the distribution
    cu2 = dict(cust_key=np.arange(0, 500, 3, dtype=np.int32))
    assert run(engine, cu2, od) == orc.q13(cu2, od, cu_key_max=499)


def test_q13_limits(engine, orc):
    od = dict(cust_key=np.zeros(1024, np.int32), comment=np.array([b"x"] * 1024, dtype="S80"))
    cu = dict(cust_key=np.arange(3, dtype=np.int32))
    with pytest.raises(capi.GpudbError) as e:      # one customer with 1024 > GPUDB_Q13_MAX_COUNT orders
        run(engine, cu, od)
    assert e.value.code == capi.E_CAPACITY
    od1 = dict(cust_key=od["cust_key"][:1023], comment=od["comment"][:1023])
    assert run(engine, cu, od1) == [(0, 2), (1023, 1)]
    with pytest.raises(capi.GpudbError) as e:
        run(engine, cu, od1, b"", b"requests")
    assert e.value.code == capi.E_INVALID
