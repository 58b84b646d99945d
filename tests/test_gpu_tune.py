"""Autotuner on the GPU: every pipeline's tuning keeps a valid setting on the context, the
results with the tuned setting equal the oracle's, and the cache round-trips."""
import ctypes as C

import pytest

from gpudbmetalbenchmark_b200 import capi
from gpudbmetalbenchmark_b200.engine import Engine, q3_to_list

pytestmark = pytest.mark.gpu


def scan_req(kind, s, **kw):
    r = capi.Request(pipeline=kind)
    r.li = C.pointer(s)
    if kind == capi.PIPE_Q6:
        r.q6 = capi.Q6Params(*kw.get("q6", (365, 730, 5, 7, 24)))
    else:
        r.q1 = capi.Q1Params(kw.get("ship_le", 2436), 0)
    return r


def test_tune_scans_then_results_match_oracle(orc):
    li = orc.lineitem(300_001, seed=19)
    with Engine(0) as e:
        t = e.upload("lineitem", li)
        s = t.lineitem()
        r6 = e.autotune(scan_req(capi.PIPE_Q6, s), reps=3)
        r1 = e.autotune(scan_req(capi.PIPE_Q1, s), reps=3)
        assert 0 <= r6["q6_variant"] <= 4 and 0 <= r1["q1_variant"] <= 10
        assert r6["candidates"] == 5 and r1["candidates"] == 11 and r6["dropped"] == 0 and r1["dropped"] == 0
        assert r6["best_ms"] <= r6["default_ms"] and r1["best_ms"] <= r1["default_ms"]
        assert e.get_option(capi.OPT_Q6_VARIANT) == r6["q6_variant"]
        assert e.get_option(capi.OPT_SCAN_VARIANT) == r1["q1_variant"]
        assert e.q6(t, 300, 1800, 2, 9, 40) == orc.q6(li, 300, 1800, 2, 9, 40)
        assert e.q1(t, 2000) == orc.q1(li, 2000)


@pytest.mark.parametrize("variant", [1, 2, 3, 4])
def test_every_q6_variant_matches_oracle(orc, variant):
    li = orc.lineitem(100_003, seed=23)
    with Engine(0) as e:
        e.set_option(capi.OPT_Q6_VARIANT, variant)
        t = e.upload("lineitem", li)
        assert e.q6(t, 100, 2000, 0, 10, 51) == orc.q6(li, 100, 2000, 0, 10, 51)


def test_tune_joins_then_results_match_oracle(orc):
    cu, od, l3 = orc.q3_tables(4000, 40_000, 160_000, 12)
    with Engine(0) as e:
        tc, to, tl = e.upload("customer", cu), e.upload("orders", od), e.upload("lineitem", l3)
        tables = capi.Q3Tables(tc.struct(), to.struct(), tl.lineitem())
        want = orc.q3(cu, od, l3, 1, 1170, 1170, 10)
        for mode, opt in ((capi.JOIN_GLOBAL, "ht_load_pct"), (capi.JOIN_RADIX, "radix_bits"),
                          (capi.JOIN_AUTO, "q3_auto_mode")):
            r = capi.Request(pipeline=capi.PIPE_Q3)
            r.q3 = C.pointer(tables)
            r.q3p = capi.Q3Params(1, 1170, 1170, 10, mode, 0)
            res = e.autotune(r, reps=2)
            assert opt in res and res["dropped"] == 0
            out = capi.Q3Result()
            e._check(e.lib.gpudb_q3_join_topk(e.ctx, C.byref(tables.cu), C.byref(tables.od), C.byref(tables.li),
                                              C.byref(r.q3p), C.byref(out), None, None))
            assert q3_to_list(out) == want
            if mode == capi.JOIN_AUTO:   # the tuned mode is what AUTO now runs
                assert res["q3_auto_mode"] in (-1, capi.JOIN_GLOBAL, capi.JOIN_RADIX, capi.JOIN_DIRECT)
                assert res["candidates"] == 4
                ran = capi.JOIN_DIRECT if res["q3_auto_mode"] == -1 else res["q3_auto_mode"]
                assert out.join_mode == ran
        e.set_option(capi.OPT_Q3_AUTO_MODE, -1)
        # every load factor gives the same answer
        for load in (50, 25):
            e.set_option(capi.OPT_HT_LOAD, load)
            assert e.q3(tc, to, tl, segment=1, order_date_lt=1170, ship_date_gt=1170, k=10) == want


def test_tune_q9(orc):
    with Engine(0) as e:
        tabs = orc.q9_tables(3000, 300, 20_000, 80_000, 4)
        ts = [e.upload(n, t) for n, t in zip(("part", "supplier", "partsupp", "orders", "lineitem"), tabs)]
        tables = capi.Q9Tables(ts[0].struct(), ts[1].struct(), ts[2].struct(), ts[3].struct(), ts[4].lineitem())
        r = capi.Request(pipeline=capi.PIPE_Q9)
        r.q9 = C.pointer(tables)
        res = e.autotune(r, reps=2)
        assert res["dropped"] == 0 and "q9_smem_slots" in res and "q9_global_slots" in res
        assert e.get_option(capi.OPT_Q9_SMEM_SLOTS) == res["q9_smem_slots"]
        assert e.q9(*ts) == orc.q9(*tabs)


def test_tune_cache_round_trip(orc, tmp_path):
    li = orc.lineitem(50_000, seed=29)
    path = tmp_path / "tune.txt"
    path.write_text("# device|pipeline|rows_log2|option|value\nsome other GPU|1|20|3|4\n")
    with Engine(0) as e:
        s = e.upload("lineitem", li).lineitem()
        r1 = e.autotune(scan_req(capi.PIPE_Q1, s), reps=2)
        r6 = e.autotune(scan_req(capi.PIPE_Q6, s), reps=2)
        e.tune_save(str(path))
    text = path.read_text()
    assert "some other GPU|1|20|3|4" in text   # other devices' lines are kept
    with Engine(0) as e2:
        assert e2.tune_load(str(path)) == 2
        assert e2.get_option(capi.OPT_SCAN_VARIANT) == r1["q1_variant"]
        assert e2.get_option(capi.OPT_Q6_VARIANT) == r6["q6_variant"]
    bad = tmp_path / "bad.txt"
    with Engine(0) as e3:
        name = text.splitlines()[-1].split("|")[0]
        bad.write_text("%s|1|20|3|99\n" % name)   # Q6 variant 99 does not exist
        with pytest.raises(capi.GpudbError) as err:
            e3.tune_load(str(bad))
        assert err.value.code == capi.E_INVALID
