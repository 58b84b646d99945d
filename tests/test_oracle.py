"""The CPU oracle against (a) the golden fixtures of an independent big-integer Python
restatement and (b) the reference's own Metal kernels compiled for the CPU
(oracle/_ref/libgpudbref.so). The reference computes in float32, so its results pin the
query logic (predicates, joins, grouping, key hashing) within float32 tolerance, and the
integer parts it computes exactly (counts, cents sums, hashes, partitions) bit-exactly."""
import json
import os

import numpy as np
import pytest

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))
LI7 = ("ship_date", "quantity", "ext_price", "discount", "tax", "flag", "status")


def need_ref(orc):
    r = orc.reference()
    if r is None:
        pytest.skip("reference kernels not built here")
    return r


# ---- golden fixtures -------------------------------------------------------------------
def test_generator_matches_golden(orc):
    for key, cols in GOLDEN["generator"].items():
        seed, off = map(int, key.split("_"))
        li = orc.lineitem(64, seed, row_offset=off)
        for name in LI7:
            assert li[name][:8].tolist() == cols[name]["head"], (key, name)
            assert int(li[name].astype(np.int64).sum()) == cols[name]["sum"], (key, name)
        ok = orc.gen(8, 64, seed, off, n_orders=50, order_mode=1)
        assert ok[:8].tolist() == cols["order_key_clustered"]["head"]
        assert int(ok.sum()) == cols["order_key_clustered"]["sum"]
        ou = orc.gen(8, 64, seed, off, n_orders=50, order_mode=2)
        assert int(ou.sum()) == cols["order_key_uniform"]["sum"]
        sk = orc.gen(10, 64, seed, off, n_parts=1000, n_supp=100)
        assert sk[:8].tolist() == cols["supp_key"]["head"]
        assert [x.decode() for x in orc.gen(34, 4, seed, off)] == cols["o_comment"]["head"], key
        for name, cid in (("commit_date", 11), ("receipt_date", 12), ("ship_mode", 13), ("o_priority", 33),
                          ("c_nation", 22), ("p_type", 42)):
            v = orc.gen(cid, 64, seed, off)
            assert v[:8].tolist() == cols[name]["head"], (key, name)
            assert int(v.astype(np.int64).sum()) == cols[name]["sum"], (key, name)


@pytest.mark.parametrize("n,seed", [(3000, 42), (2500, 9)])
def test_q6_q1_match_golden(orc, n, seed):
    li = orc.lineitem(n, seed)
    assert list(orc.q6(li)) == GOLDEN["q6"]["%d_%d" % (n, seed)]
    assert list(orc.q6(li, 0, 2527, 0, 10, 51)) == GOLDEN["q6"]["%d_%d_wide" % (n, seed)]
    for cut, tag in ((2436, ""), (100, "_cut100")):
        got = orc.q1(li, cut)
        want = GOLDEN["q1"]["%d_%d%s" % (n, seed, tag)]
        assert sorted("%d%d" % k for k in got) == sorted(want)
        for k, g in got.items():
            w = [int(x) for x in want["%d%d" % k]]
            assert [g["count"], g["sum_qty"], g["sum_base_price"], g["sum_disc_price"], g["sum_charge"],
                    g["sum_discount"]] == w


def test_q3_matches_golden(orc):
    cu, od, li = orc.q3_tables(300, 1200, 4800, 42)
    top, groups = orc.q3(cu, od, li)
    want = GOLDEN["q3"]["300_1200_4800_42"]
    assert groups == want["groups"]
    assert [[a, b, str(c)] for a, b, c in top] == want["top"]
    cu, od, li = orc.q3_tables(200, 900, 3000, 5)
    top, groups = orc.q3(cu, od, li, segment=3, date_lt=2000, ship_gt=300, k=20)
    want = GOLDEN["q3"]["200_900_3000_5_seg3"]
    assert groups == want["groups"]
    assert [[a, b, str(c)] for a, b, c in top] == want["top"]


def test_q9_matches_golden(orc):
    tabs = orc.q9_tables(400, 40, 1500, 6000, 42)
    rows, n = orc.q9(*tabs)
    assert [[a, b, str(c)] for a, b, c in rows] == GOLDEN["q9"]["400_40_1500_6000_42"]
    assert n == len(rows)


def test_q4_q12_match_golden(orc):
    od, li = orc.q4_tables(3000, 12000, 42)
    assert orc.q4(od, li) == GOLDEN["q4"]["3000_12000_42"]
    assert orc.q12(od, li) == [tuple(x) for x in GOLDEN["q12"]["3000_12000_42"]]
    od, li = orc.q4_tables(2000, 9000, 5)
    assert orc.q4(od, li, 0, 2406) == GOLDEN["q4"]["2000_9000_5_wide"]
    assert orc.q12(od, li, 0, 2600, (0, 6), 3) == [tuple(x) for x in GOLDEN["q12"]["2000_9000_5_air_truck_hi3"]]


def test_q13_matches_golden(orc):
    cu, od = orc.q13_tables(300, 3000, 42)
    assert orc.q13(cu, od) == [tuple(x) for x in GOLDEN["q13"]["300_3000_42"]]
    cu, od = orc.q13_tables(200, 4000, 9)
    assert orc.q13(cu, od, b"pinto", b"beans") == [tuple(x) for x in GOLDEN["q13"]["200_4000_9_pinto_beans"]]


EUROPE = (1 << 6) | (1 << 7) | (1 << 19) | (1 << 22) | (1 << 23)


def test_q5_matches_golden(orc):
    cu, su, od, li = orc.q5_tables(300, 40, 3000, 12000, 42)
    assert orc.q5(cu, su, od, li) == [(n, int(r)) for n, r in GOLDEN["q5"]["300_40_3000_12000_42"]]
    cu, su, od, li = orc.q5_tables(500, 60, 4000, 16000, 3)
    assert orc.q5(cu, su, od, li, 0, 2406, EUROPE) == \
        [(n, int(r)) for n, r in GOLDEN["q5"]["500_60_4000_16000_3_europe_all_years"]]


@pytest.mark.parametrize("sizes,seed,window,mask", [((300, 40, 3000, 12000), 42, (731, 1096), None),
                                                    ((3000, 200, 30000, 120000), 7, (0, 2406), EUROPE)])
def test_q5_pinned_to_reference_kernels(orc, sizes, seed, window, mask):
    """Q5 revenue per nation against the reference's kernels (float32 there: within its
    tolerance; which nations have revenue, exactly)."""
    ref = need_ref(orc)
    cu, su, od, li = orc.q5_tables(*sizes, seed)
    mask = orc.ASIA if mask is None else mask
    mine = np.zeros(25, np.int64)
    orc.q5(cu, su, od, li, *window, mask, revenue_out=mine)
    theirs = np.zeros(25, np.float32)
    ref.ref_q5(len(cu["cust_key"]), cu["cust_key"].ctypes.data, cu["nation"].ctypes.data, len(su["supp_key"]),
               su["supp_key"].ctypes.data, su["nation"].ctypes.data, len(od["order_key"]), od["order_key"].ctypes.data,
               od["cust_key"].ctypes.data, od["order_date"].ctypes.data, len(li["order_key"]),
               li["order_key"].ctypes.data, li["supp_key"].ctypes.data, li["ext_price"].ctypes.data,
               li["discount"].ctypes.data, *window, mask, 8, 4, theirs.ctypes.data)
    assert np.array_equal(mine > 0, theirs > 0)
    np.testing.assert_allclose(theirs, mine / 10000.0, rtol=1e-4)


ASIA = (1 << 8) | (1 << 9) | (1 << 12) | (1 << 18) | (1 << 21)


def test_q7_q8_match_golden(orc):
    t = orc.q8_tables(400, 40, 600, 3000, 12000, 42)
    assert orc.q7(t[0], t[1], t[3], t[4]) == [tuple(r[:3]) + (int(r[3]),) for r in GOLDEN["q7"]["400_40_600_3000_12000_42"]]
    t = orc.q8_tables(400, 40, 600, 3000, 12000, 5)
    assert orc.q7(t[0], t[1], t[3], t[4], 17, 18, 0, 2556) == \
        [tuple(r[:3]) + (int(r[3]),) for r in GOLDEN["q7"]["400_40_600_3000_12000_5_peru_china_all"]]
    t = orc.q8_tables(400, 40, 300, 3000, 12000, 42)
    assert orc.q8(*t, part_type=7) == [(y, int(a), int(b)) for y, a, b in GOLDEN["q8"]["400_40_300_3000_12000_42_type7"]]
    t = orc.q8_tables(500, 40, 300, 4000, 16000, 9)
    assert orc.q8(*t, 12, ASIA, 103, 366, 2191) == \
        [(y, int(a), int(b)) for y, a, b in GOLDEN["q8"]["500_40_300_4000_16000_9_japan_asia_1993_1997"]]


@pytest.mark.parametrize("sizes,seed", [((400, 40, 600, 3000, 12000), 42), ((5000, 400, 8000, 50000, 200000), 7)])
def test_q7_pinned_to_reference_kernels(orc, sizes, seed):
    """Q7 bins (FRANCE/GERMANY, 1995-1996: the years the reference's kernel bins) against its
    kernels, within float32 tolerance; which bins are nonzero, exactly."""
    ref = need_ref(orc)
    cu, su, pa, od, li = orc.q8_tables(*sizes, seed)
    mine = {(s, y): r for s, c, y, r in orc.q7(cu, su, od, li)}
    bins = np.zeros(4, np.float32)
    ref.ref_q7(len(cu["cust_key"]), cu["cust_key"].ctypes.data, cu["nation"].ctypes.data, len(su["supp_key"]),
               su["supp_key"].ctypes.data, su["nation"].ctypes.data, len(od["order_key"]), od["order_key"].ctypes.data,
               od["cust_key"].ctypes.data, len(li["order_key"]), li["order_key"].ctypes.data, li["supp_key"].ctypes.data,
               li["ship_date"].ctypes.data, li["ext_price"].ctypes.data, li["discount"].ctypes.data, orc.FRANCE,
               orc.GERMANY, 1096, 1826, 8, 4, bins.ctypes.data)
    want = np.array([mine.get((orc.FRANCE, 1995), 0), mine.get((orc.FRANCE, 1996), 0),
                     mine.get((orc.GERMANY, 1995), 0), mine.get((orc.GERMANY, 1996), 0)], np.float64) / 10000.0
    assert np.array_equal(bins > 0, want > 0)
    np.testing.assert_allclose(bins, want, rtol=1e-4)


@pytest.mark.parametrize("sizes,seed,ptype", [((3000, 200, 2000, 30000, 120000), 42, 103),
                                              ((5000, 400, 1000, 50000, 200000), 7, 7)])
def test_q8_pinned_to_reference_kernels(orc, sizes, seed, ptype):
    """Q8 per-year nation and total volume (BRAZIL in AMERICA, 1995-1996) against the reference's
    kernels, within float32 tolerance."""
    ref = need_ref(orc)
    cu, su, pa, od, li = orc.q8_tables(*sizes, seed)
    mine = orc.q8(cu, su, pa, od, li, part_type=ptype)
    bins = np.zeros(4, np.float32)
    ref.ref_q8(len(cu["cust_key"]), cu["cust_key"].ctypes.data, cu["nation"].ctypes.data, len(su["supp_key"]),
               su["supp_key"].ctypes.data, su["nation"].ctypes.data, len(pa["part_key"]), pa["part_key"].ctypes.data,
               pa["type"].ctypes.data, len(od["order_key"]), od["order_key"].ctypes.data, od["cust_key"].ctypes.data,
               od["order_date"].ctypes.data, len(li["order_key"]), li["order_key"].ctypes.data,
               li["part_key"].ctypes.data, li["supp_key"].ctypes.data, li["ext_price"].ctypes.data,
               li["discount"].ctypes.data, 1096, 1826, orc.AMERICA, orc.BRAZIL, ptype, 8, 4, bins.ctypes.data)
    want = np.array([mine[0][1], mine[1][1], mine[0][2], mine[1][2]], np.float64) / 10000.0
    assert want[2] > 0 and np.array_equal(bins > 0, want > 0)
    np.testing.assert_allclose(bins, want, rtol=1e-4)


def test_q10_matches_golden(orc):
    cu, od, li = orc.q10_tables(300, 3000, 12000, 42)
    g = GOLDEN["q10"]["300_3000_12000_42"]
    assert orc.q10(cu, od, li) == ([(c, int(r)) for c, r in g["top"]], g["customers"])
    cu, od, li = orc.q10_tables(200, 2000, 9000, 5)
    g = GOLDEN["q10"]["200_2000_9000_5_wide"]
    assert orc.q10(cu, od, li, 0, 2406, 7) == ([(c, int(r)) for c, r in g["top"]], g["customers"])


def test_q1_q6_threaded_equal_serial(orc):
    li = orc.lineitem(50_000, 3)
    assert orc.q6(li) == orc.q6(li, threads=4)
    assert orc.q1(li) == orc.q1(li, threads=3)


# ---- the reference's own kernels -----------------------------------------------------------
@pytest.mark.parametrize("n,seed,params", [(20000, 42, (365, 730, 5, 7, 24)), (7777, 3, (0, 2527, 0, 10, 51)),
                                           (5000, 11, (1000, 1400, 2, 9, 40))])
def test_q6_pinned_to_reference_kernel(orc, n, seed, params):
    ref = need_ref(orc)
    li = orc.lineitem(n, seed)
    rev, m = orc.q6(li, *params)
    p = li
    got = ref.ref_q6(n, p["ship_date"].ctypes.data, p["discount"].ctypes.data, p["quantity"].ctypes.data,
                     p["ext_price"].ctypes.data, *params, 64, 4)
    # reference revenue is in dollars (ext / 100 * disc / 100), summed in float32
    assert got == pytest.approx(rev / 10000.0, rel=2e-5, abs=1e-2)


@pytest.mark.parametrize("n,seed,cut", [(20000, 42, 2436), (3001, 8, 500), (4000, 1, 2526)])
def test_q1_pinned_to_reference_kernel(orc, n, seed, cut):
    ref = need_ref(orc)
    li = orc.lineitem(n, seed)
    out = np.zeros(36, np.int64)
    ref.ref_q1(n, *(li[c].ctypes.data for c in LI7), cut, 32, 4, out.ctypes.data)
    mine = orc.q1(li, cut)
    for b in range(6):
        o = out[b * 6:(b + 1) * 6]
        g = mine.get((b // 2, b % 2))
        if g is None:
            assert o[5] == 0
            continue
        # exact in the reference: counts, quantity cents, discount points
        c = g["count"]
        assert o[5] == c
        assert o[0] == g["sum_qty"] * 100
        assert o[4] == g["sum_discount"]
        # float32 prices: the reference's cents recovery floor(x*100+0.5) can be off by one
        # cent per row; disc_price and charge are then rounded to cents per row
        # (kernels/q1.metal:84-89): at most 1.5 and 2.12 cents per row
        assert abs(o[1] - g["sum_base_price"]) <= c
        assert abs(o[2] * 100 - g["sum_disc_price"]) <= 150 * c
        assert abs(o[3] * 10000 - g["sum_charge"]) <= 21200 * c
        # and the totals agree to 1e-6 relative
        assert o[3] * 10000 == pytest.approx(g["sum_charge"], rel=1e-6)


@pytest.mark.parametrize("sizes,seed,params", [((300, 1200, 4800), 42, (1, 1170, 1170)),
                                               ((500, 3000, 12000), 7, (3, 2000, 400))])
def test_q3_pinned_to_reference_kernels(orc, sizes, seed, params):
    ref = need_ref(orc)
    cu, od, li = orc.q3_tables(*sizes, seed)
    top, groups = orc.q3(cu, od, li, *params, k=100000)
    cap = 1 << 16
    gk, gr, gd = np.zeros(cap, np.int32), np.zeros(cap, np.float32), np.zeros(cap, np.int32)
    n = ref.ref_q3(len(cu["cust_key"]), cu["cust_key"].ctypes.data, cu["segment"].ctypes.data,
                   len(od["order_key"]), od["order_key"].ctypes.data, od["cust_key"].ctypes.data,
                   od["order_date"].ctypes.data, len(li["order_key"]), li["order_key"].ctypes.data,
                   li["ship_date"].ctypes.data, li["ext_price"].ctypes.data, li["discount"].ctypes.data,
                   *params, 16, 4, gk.ctypes.data, gr.ctypes.data, gd.ctypes.data, cap)
    assert n == groups
    theirs = {int(gk[i]): (float(gr[i]), int(gd[i])) for i in range(n)}
    mine = {k: (r, d) for k, d, r in top}
    assert set(theirs) == set(mine)
    for k, (r, d) in mine.items():
        assert theirs[k][1] == d
        assert theirs[k][0] == pytest.approx(r / 10000.0, rel=1e-5)


def test_q9_pinned_to_reference_kernels(orc):
    ref = need_ref(orc)
    pa, su, ps, od, li = orc.q9_tables(2000, 100, 3000, 40000, 5)
    mine, n = orc.q9(pa, su, ps, od, li)
    cap = 512
    gn, gy, gp = np.zeros(cap, np.int32), np.zeros(cap, np.int32), np.zeros(cap, np.float32)
    m = ref.ref_q9(len(pa["part_key"]), pa["part_key"].ctypes.data, pa["flag"].ctypes.data,
                   len(su["supp_key"]), su["supp_key"].ctypes.data, su["nation"].ctypes.data,
                   len(ps["part_key"]), ps["part_key"].ctypes.data, ps["supp_key"].ctypes.data,
                   ps["supply_cost"].ctypes.data, len(od["order_key"]), od["order_key"].ctypes.data,
                   od["order_date"].ctypes.data, len(li["part_key"]), li["part_key"].ctypes.data,
                   li["supp_key"].ctypes.data, li["order_key"].ctypes.data, li["ext_price"].ctypes.data,
                   li["discount"].ctypes.data, li["quantity"].ctypes.data, 8, 4,
                   gn.ctypes.data, gy.ctypes.data, gp.ctypes.data, cap)
    assert m == n
    theirs = {(int(gn[i]), int(gy[i])): float(gp[i]) for i in range(m)}
    assert set(theirs) == {(a, b) for a, b, _ in mine}
    for a, b, p in mine:
        assert theirs[(a, b)] == pytest.approx(p / 10000.0, rel=1e-4, abs=1.0)


@pytest.mark.parametrize("n_or,n_li,seed,window", [(3000, 12000, 42, (547, 639)), (20000, 90000, 7, (0, 2406)),
                                                    (5000, 20000, 3, (1500, 1530))])
def test_q4_pinned_to_reference_kernels(orc, n_or, n_li, seed, window):
    """Q4 counts are integers in the reference too: bit-exact against its kernels."""
    ref = need_ref(orc)
    od, li = orc.q4_tables(n_or, n_li, seed)
    out = np.zeros(5, np.uint32)
    ref.ref_q4(n_or, od["order_key"].ctypes.data, od["order_date"].ctypes.data, od["priority"].ctypes.data, n_li,
               li["order_key"].ctypes.data, li["commit_date"].ctypes.data, li["receipt_date"].ctypes.data, *window,
               16, 4, out.ctypes.data)
    assert orc.q4(od, li, *window) == out.tolist()


@pytest.mark.parametrize("n_or,n_li,seed,window", [(3000, 12000, 42, (731, 1096)), (20000, 90000, 7, (0, 2600)),
                                                    (5000, 20000, 3, (900, 960))])
def test_q12_pinned_to_reference_kernels(orc, n_or, n_li, seed, window):
    """Q12 with the query's modes (MAIL, SHIP) and priorities ('1-URGENT', '2-HIGH'): bit-exact
    against the reference's kernels (bins MAIL high, MAIL low, SHIP high, SHIP low)."""
    ref = need_ref(orc)
    od, li = orc.q4_tables(n_or, n_li, seed)
    out = np.zeros(4, np.uint32)
    ref.ref_q12(n_or, od["order_key"].ctypes.data, od["priority"].ctypes.data, n_li, li["order_key"].ctypes.data,
                li["ship_date"].ctypes.data, li["commit_date"].ctypes.data, li["receipt_date"].ctypes.data,
                li["ship_mode"].ctypes.data, *window, 16, 4, out.ctypes.data)
    (mh, ml), (sh, sl) = orc.q12(od, li, *window)
    assert [mh, ml, sh, sl] == out.tolist()


@pytest.mark.parametrize("n_cu,n_or,seed", [(300, 3000, 42), (5000, 60000, 7)])
def test_q13_pinned_to_reference_kernels(orc, n_cu, n_or, seed):
    """Q13's pattern match, counts and histogram are integer work in the reference too:
    bit-exact against its kernels (the reference keeps 256 bins)."""
    ref = need_ref(orc)
    cu, od = orc.q13_tables(n_cu, n_or, seed)
    hist = np.zeros(256, np.uint32)
    ref.ref_q13(n_cu, n_or, od["cust_key"].ctypes.data, od["comment"].ctypes.data, 8, 4, hist.ctypes.data)
    theirs = sorted(((c, int(d)) for c, d in enumerate(hist) if d), key=lambda x: (-x[1], -x[0]))
    assert orc.q13(cu, od) == theirs


@pytest.mark.parametrize("sizes,seed,window", [((300, 3000, 12000), 42, (639, 731)), ((2000, 20000, 80000), 7, (0, 2406))])
def test_q10_pinned_to_reference_kernels(orc, sizes, seed, window):
    """Q10 per-customer revenue against the reference's kernels (float32 there: within its
    tolerance; which customers have revenue, exactly)."""
    ref = need_ref(orc)
    cu, od, li = orc.q10_tables(*sizes, seed)
    n_cu = sizes[0]
    mine = np.zeros(n_cu, np.int64)
    orc.q10(cu, od, li, *window, rev_out=mine)
    theirs = np.zeros(n_cu, np.float32)
    ref.ref_q10(len(od["order_key"]), od["order_key"].ctypes.data, od["cust_key"].ctypes.data,
                od["order_date"].ctypes.data, len(li["order_key"]), li["order_key"].ctypes.data, li["flag"].ctypes.data,
                li["ext_price"].ctypes.data, li["discount"].ctypes.data, *window, 8, 4, theirs.ctypes.data, n_cu)
    assert np.array_equal(mine > 0, theirs > 0)
    np.testing.assert_allclose(theirs, mine / 10000.0, rtol=1e-4)


def test_micro_pinned_to_reference_kernels(orc):
    ref = need_ref(orc)
    col = orc.gen(1, 10000, 4)
    for v in (0, 100, 1000, 2527, 3000):
        c, bits, rows = orc.select_lt(col, v)
        words = np.zeros(len(col), np.uint32)
        ref.ref_select_lt(len(col), col.ctypes.data, v, words.ctypes.data)
        assert int(words.sum()) == c
        assert np.array_equal(np.nonzero(words)[0].astype(np.uint32), rows)
    q = orc.gen(2, 10000, 4)
    assert ref.ref_sum(len(q), q.ctypes.data, 16, 4) == pytest.approx(orc.sum_i32(q), rel=1e-6)
    b = orc.gen(30, 1500, 4)
    p = orc.gen(8, 6000, 4, n_orders=1700, order_mode=2)
    assert ref.ref_join_count(len(b), b.ctypes.data, len(p), p.ctypes.data) == orc.join_count(b, p)


def test_radix_partition_pinned_to_reference_kernels(orc):
    ref = need_ref(orc)
    keys = orc.gen(8, 20000, 6, n_orders=50000, order_mode=2)
    pay = np.arange(len(keys), dtype=np.int32)
    hist, off = np.zeros(1024, np.uint32), np.zeros(1024, np.uint32)
    ko, po = np.zeros(len(keys), np.int32), np.zeros(len(keys), np.int32)
    ref.ref_radix_partition(len(keys), keys.ctypes.data, pay.ctypes.data, hist.ctypes.data, off.ctypes.data,
                            ko.ctypes.data, po.ctypes.data)
    mko, mpo, moff = orc.radix_partition(keys, pay, 10)
    assert np.array_equal(moff[:1024], off)
    assert np.array_equal(np.diff(moff), hist)
    # the single-thread reference scatter keeps input order, like the oracle's partition
    assert np.array_equal(ko, mko) and np.array_equal(po, mpo)
    assert all(orc.oracle().or_key_hash(int(k)) & 1023 == p for p in range(0, 1024, 97)
               for k in mko[moff[p]:moff[p + 1]])


def test_partition_join_pinned_to_reference_kernel(orc):
    ref = need_ref(orc)
    b = orc.gen(8, 3000, 2, n_orders=4000, order_mode=2)   # duplicates included
    p = orc.gen(8, 9000, 3, n_orders=4000, order_mode=2)
    cap = 200000
    ob, op = np.zeros(cap, np.int32), np.zeros(cap, np.int32)
    n = ref.ref_partition_join(len(b), b.ctypes.data, len(p), p.ctypes.data, ob.ctypes.data, op.ctypes.data, cap)
    mb, mp, mn = orc.join_pairs(b, p, cap)
    assert n == mn
    assert sorted(zip(op[:n].tolist(), ob[:n].tolist())) == sorted(zip(mp.tolist(), mb.tolist()))
