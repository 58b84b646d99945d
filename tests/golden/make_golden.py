"""Writes tests/golden/golden.json: small seeded cases computed by an independent
pure-Python (big-integer) restatement of the synthetic generator and of each pipeline.
The oracle (oracle/oracle.c) and the engine are checked against these values.

    python tests/golden/make_golden.py
"""
import json
import os

M64 = (1 << 64) - 1
G = 0x9E3779B97F4A7C15


def fin(z):
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def stream(seed, col):
    return fin((seed * G + (col + 1) * 0xD1B54A32D192ED03) & M64)


def uniform(key, row, lo, hi):
    v = fin((key + (row + 1) * G) & M64)
    return lo + ((v * (hi - lo + 1)) >> 64)


def column(name, n, seed, off=0, n_orders=0, n_cust=0, n_parts=0, n_supp=0, mode=0):
    k = lambda s: stream(seed, s)  # noqa: E731
    rows = range(off, off + n)
    if name == "ship_date":
        return [uniform(k(16), r, 0, 2526) for r in rows]
    if name == "quantity":
        return [uniform(k(17), r, 1, 50) for r in rows]
    if name == "ext_price":
        return [uniform(k(17), r, 1, 50) * uniform(k(18), r, 90000, 209900) for r in rows]
    if name == "discount":
        return [uniform(k(19), r, 0, 10) for r in rows]
    if name == "tax":
        return [uniform(k(20), r, 0, 8) for r in rows]
    if name == "flag":
        return [uniform(k(21), r, 0, 2) for r in rows]
    if name == "status":
        return [uniform(k(22), r, 0, 1) for r in rows]
    if name == "order_key":
        if mode == 2:
            return [4 * uniform(k(23), r, 0, n_orders - 1) + 1 for r in rows]
        out, s = [], 0
        while len(out) < off + n:
            out += [4 * (s % n_orders) + 1] * uniform(k(26), s, 1, 7)
            s += 1
        return out[off:off + n]
    if name == "part_key":
        return [uniform(k(24), r, 0, n_parts - 1) for r in rows]
    if name == "supp_key":
        return [(uniform(k(24), r, 0, n_parts - 1) + uniform(k(25), r, 0, 3) * (n_supp // 4)) % n_supp for r in rows]
    if name == "commit_date":
        return [uniform(k(16), r, 0, 2526) + uniform(k(27), r, -91, 89) for r in rows]
    if name == "receipt_date":
        return [uniform(k(16), r, 0, 2526) + uniform(k(28), r, 1, 30) for r in rows]
    if name == "ship_mode":
        return [uniform(k(29), r, 0, 6) for r in rows]
    if name == "o_priority":
        return [uniform(k(50), r, 1, 5) for r in rows]
    if name == "o_comment":
        vocab = ("special requests packages deposits accounts instructions foxes ideas theodolites pinto beans "
                 "platelets furiously carefully quickly slyly blithely regular final pending ironic express bold "
                 "even").split()
        out = []
        for r in rows:
            words, text = uniform(k(51), r * 16, 2, 9), ""
            for i in range(words):
                w = vocab[uniform(k(51), r * 16 + 1 + i, 0, 23)]
                nxt = (text + " " + w) if text else w
                if len(nxt) > 79:
                    break
                text = nxt
            out.append(text)
        return out
    if name == "p_type":
        return [uniform(k(65), r, 0, 149) for r in rows]
    if name == "c_nation":
        return [uniform(k(33), r, 0, 24) for r in rows]
    if name == "segment":
        return [uniform(k(32), r, 0, 4) for r in rows]
    if name == "o_cust":
        return [uniform(k(48), r, 0, n_cust - 1) for r in rows]
    if name == "o_date":
        return [uniform(k(49), r, 0, 2405) for r in rows]
    if name == "p_flag":
        return [1 if uniform(k(64), r, 0, 999) < 55 else 0 for r in rows]
    if name == "nation":
        return [uniform(k(80), r, 0, 24) for r in rows]
    if name == "ps_cost":
        return [uniform(k(96), r, 100, 100000) for r in rows]
    raise KeyError(name)


def q6(li, lo=365, hi=730, dlo=5, dhi=7, qlt=24):
    rev = cnt = 0
    for s, d, q, e in zip(li["ship_date"], li["discount"], li["quantity"], li["ext_price"]):
        if lo <= s < hi and dlo <= d <= dhi and q < qlt:
            rev += e * d
            cnt += 1
    return [rev, cnt]


def q1(li, ship_le=2436):
    g = {}
    for s, q, e, d, t, f, st in zip(*(li[c] for c in ("ship_date", "quantity", "ext_price", "discount", "tax",
                                                       "flag", "status"))):
        if s > ship_le:
            continue
        a = g.setdefault("%d%d" % (f, st), [0, 0, 0, 0, 0, 0])
        a[0] += 1
        a[1] += q
        a[2] += e
        a[3] += e * (100 - d)
        a[4] += e * (100 - d) * (100 + t)
        a[5] += d
    return {k: [str(x) for x in v] for k, v in sorted(g.items())}


def q3(n_cu, n_or, n_li, seed, segment=1, date_lt=1170, ship_gt=1170, k=10):
    seg = column("segment", n_cu, seed)
    ocust = column("o_cust", n_or, seed, n_cust=n_cu)
    odate = column("o_date", n_or, seed)
    okey = [4 * i + 1 for i in range(n_or)]
    li = {c: column(c, n_li, seed, n_orders=n_or, mode=1) for c in ("order_key", "ship_date", "ext_price", "discount")}
    good = {okey[i]: odate[i] for i in range(n_or) if odate[i] < date_lt and seg[ocust[i]] == segment}
    rev = {}
    for key, s, e, d in zip(li["order_key"], li["ship_date"], li["ext_price"], li["discount"]):
        if s > ship_gt and key in good:
            rev[key] = rev.get(key, 0) + e * (100 - d)
    rows = sorted(((key, good[key], r) for key, r in rev.items()), key=lambda x: (-x[2], x[1], x[0]))
    return {"groups": len(rows), "top": [[a, b, str(c)] for a, b, c in rows[:k]]}


def q9(n_pa, n_su, n_or, n_li, seed):
    pflag = column("p_flag", n_pa, seed)
    nation = column("nation", n_su, seed)
    cost = column("ps_cost", 4 * n_pa, seed)
    pscost = {(r // 4, (r // 4 + (r % 4) * (n_su // 4)) % n_su): cost[r] for r in range(4 * n_pa)}
    odate = column("o_date", n_or, seed)
    year = {4 * i + 1: 1992 + odate[i] // 365 for i in range(n_or)}
    li = {c: column(c, n_li, seed, n_orders=n_or, n_parts=n_pa, n_supp=n_su, mode=2)
          for c in ("part_key", "supp_key", "order_key", "ext_price", "discount", "quantity")}
    g = {}
    for p, s, o, e, d, q in zip(*(li[c] for c in ("part_key", "supp_key", "order_key", "ext_price", "discount",
                                                   "quantity"))):
        if not pflag[p] or (p, s) not in pscost or o not in year:
            continue
        key = (nation[s], year[o])
        g[key] = g.get(key, 0) + e * (100 - d) - pscost[(p, s)] * q * 100
    rows = sorted(g.items(), key=lambda kv: (kv[0][0], -kv[0][1]))
    return [[a, b, str(v)] for (a, b), v in rows]


def q4_q12_tables(n_or, n_li, seed):
    od = {"order_key": [4 * i + 1 for i in range(n_or)], "order_date": column("o_date", n_or, seed),
          "priority": column("o_priority", n_or, seed)}
    li = {c: column(c, n_li, seed, n_orders=n_or, mode=1)
          for c in ("order_key", "ship_date", "commit_date", "receipt_date", "ship_mode")}
    return od, li


def q4(n_or, n_li, seed, date_lo=547, date_hi=639):
    od, li = q4_q12_tables(n_or, n_li, seed)
    late = {k for k, c, r in zip(li["order_key"], li["commit_date"], li["receipt_date"]) if c < r}
    cnt = [0] * 5
    for k, d, p in zip(od["order_key"], od["order_date"], od["priority"]):
        if date_lo <= d < date_hi and k in late:
            cnt[p - 1] += 1
    return cnt


def q12(n_or, n_li, seed, receipt_lo=731, receipt_hi=1096, modes=(2, 5), high_max=2):
    od, li = q4_q12_tables(n_or, n_li, seed)
    high = {k for k, p in zip(od["order_key"], od["priority"]) if 1 <= p <= high_max}
    out = [[0, 0], [0, 0]]
    for k, s, c, r, m in zip(*(li[x] for x in ("order_key", "ship_date", "commit_date", "receipt_date",
                                                "ship_mode"))):
        if m not in modes or not (receipt_lo <= r < receipt_hi) or c >= r or s >= c:
            continue
        out[modes.index(m)][0 if k in high else 1] += 1
    return out


def q13(n_cu, n_or, seed, w1="special", w2="requests"):
    cust = column("o_cust", n_or, seed, n_cust=n_cu)
    comment = column("o_comment", n_or, seed)
    cnt = [0] * n_cu
    for c, t in zip(cust, comment):
        a = t.find(w1)
        if a < 0 or t.find(w2, a + len(w1)) < 0:
            cnt[c] += 1
    hist = {}
    for v in cnt:
        hist[v] = hist.get(v, 0) + 1
    return sorted(([c, d] for c, d in hist.items()), key=lambda x: (-x[1], -x[0]))


def q5(n_cu, n_su, n_or, n_li, seed, date_lo=731, date_hi=1096, nations=(8, 9, 12, 18, 21)):
    cnat = column("c_nation", n_cu, seed)
    snat = column("nation", n_su, seed)
    ocust = column("o_cust", n_or, seed, n_cust=n_cu)
    odate = column("o_date", n_or, seed)
    onat = {4 * i + 1: cnat[ocust[i]] for i in range(n_or) if date_lo <= odate[i] < date_hi and cnat[ocust[i]] in nations}
    li = {c: column(c, n_li, seed, n_orders=n_or, n_parts=n_su * 20, n_supp=n_su, mode=1)
          for c in ("order_key", "supp_key", "ext_price", "discount")}
    rev = {}
    for key, sk, e, d in zip(li["order_key"], li["supp_key"], li["ext_price"], li["discount"]):
        if key in onat and snat[sk] == onat[key]:
            rev[onat[key]] = rev.get(onat[key], 0) + e * (100 - d)
    return [[n, str(r)] for n, r in sorted(rev.items(), key=lambda x: (-x[1], x[0])) if r]


NATIONS = ("ALGERIA", "ARGENTINA", "BRAZIL", "CANADA", "EGYPT", "ETHIOPIA", "FRANCE", "GERMANY", "INDIA", "INDONESIA",
           "IRAN", "IRAQ", "JAPAN", "JORDAN", "KENYA", "MOROCCO", "MOZAMBIQUE", "PERU", "CHINA", "ROMANIA",
           "SAUDI ARABIA", "VIETNAM", "RUSSIA", "UNITED KINGDOM", "UNITED STATES")


def year_of_day(d):
    y = 1992
    ylen = lambda y: 366 if (y % 4 == 0 and y % 100 != 0) or y % 400 == 0 else 365  # noqa: E731
    while d < 0:
        y -= 1
        d += ylen(y)
    while d >= ylen(y):
        d -= ylen(y)
        y += 1
    return y


def q7q8_tables(n_cu, n_su, n_pa, n_or, n_li, seed):
    t = {"c_nation": column("c_nation", n_cu, seed), "s_nation": column("nation", n_su, seed),
         "p_type": column("p_type", n_pa, seed), "o_cust": column("o_cust", n_or, seed, n_cust=n_cu),
         "o_date": column("o_date", n_or, seed)}
    t["li"] = {c: column(c, n_li, seed, n_orders=n_or, n_parts=n_pa, n_supp=n_su, mode=1)
               for c in ("order_key", "part_key", "supp_key", "ship_date", "ext_price", "discount")}
    return t


def q7(n_cu, n_su, n_pa, n_or, n_li, seed, a=6, b=7, lo=1096, hi=1826):
    t = q7q8_tables(n_cu, n_su, n_pa, n_or, n_li, seed)
    cust_nation = {4 * i + 1: t["c_nation"][t["o_cust"][i]] for i in range(n_or)}
    rev = {}
    li = t["li"]
    for key, sk, sd, e, d in zip(li["order_key"], li["supp_key"], li["ship_date"], li["ext_price"], li["discount"]):
        if not lo <= sd <= hi:
            continue
        s, c = t["s_nation"][sk], cust_nation[key]
        if (s, c) in ((a, b), (b, a)):
            g = (s, c, year_of_day(sd))
            rev[g] = rev.get(g, 0) + e * (100 - d)
    order = sorted(rev.items(), key=lambda kv: (NATIONS[kv[0][0]], NATIONS[kv[0][1]], kv[0][2]))
    return [[s, c, y, str(r)] for (s, c, y), r in order if r]


def q8(n_cu, n_su, n_pa, n_or, n_li, seed, nation=2, region=(1, 2, 3, 17, 24), ptype=103, lo=1096, hi=1826):
    t = q7q8_tables(n_cu, n_su, n_pa, n_or, n_li, seed)
    year = {4 * i + 1: year_of_day(t["o_date"][i]) for i in range(n_or)
            if lo <= t["o_date"][i] <= hi and t["c_nation"][t["o_cust"][i]] in region}
    vol, nvol = {}, {}
    li = t["li"]
    for key, pk, sk, e, d in zip(li["order_key"], li["part_key"], li["supp_key"], li["ext_price"], li["discount"]):
        if t["p_type"][pk] != ptype or key not in year:
            continue
        y = year[key]
        vol[y] = vol.get(y, 0) + e * (100 - d)
        if t["s_nation"][sk] == nation:
            nvol[y] = nvol.get(y, 0) + e * (100 - d)
    return [[y, str(nvol.get(y, 0)), str(vol.get(y, 0))] for y in range(year_of_day(lo), year_of_day(hi) + 1)]


def q10(n_cu, n_or, n_li, seed, date_lo=639, date_hi=731, k=20):
    ocust = column("o_cust", n_or, seed, n_cust=n_cu)
    odate = column("o_date", n_or, seed)
    cust_of = {4 * i + 1: ocust[i] for i in range(n_or) if date_lo <= odate[i] < date_hi}
    li = {c: column(c, n_li, seed, n_orders=n_or, mode=1) for c in ("order_key", "flag", "ext_price", "discount")}
    rev = {}
    for key, f, e, d in zip(li["order_key"], li["flag"], li["ext_price"], li["discount"]):
        if f == 2 and key in cust_of:
            rev[cust_of[key]] = rev.get(cust_of[key], 0) + e * (100 - d)
    rows = sorted(((c, r) for c, r in rev.items() if r > 0), key=lambda x: (-x[1], x[0]))
    return {"customers": len(rows), "top": [[c, str(r)] for c, r in rows[:k]]}


def main():
    out = {"generator": {}, "q6": {}, "q1": {}, "q3": {}, "q9": {}, "q4": {}, "q12": {}, "q13": {}, "q10": {}, "q5": {}, "q7": {}, "q8": {}}
    # generator: first values and column sums for two seeds and a shifted window
    for seed, off in ((42, 0), (7, 1000)):
        cols = {}
        for name in ("ship_date", "quantity", "ext_price", "discount", "tax", "flag", "status"):
            v = column(name, 64, seed, off)
            cols[name] = {"head": v[:8], "sum": sum(v)}
        for name in ("order_key",):
            v1 = column(name, 64, seed, off, n_orders=50, mode=1)
            v2 = column(name, 64, seed, off, n_orders=50, mode=2)
            cols["order_key_clustered"] = {"head": v1[:8], "sum": sum(v1)}
            cols["order_key_uniform"] = {"head": v2[:8], "sum": sum(v2)}
        v = column("supp_key", 64, seed, off, n_parts=1000, n_supp=100)
        cols["supp_key"] = {"head": v[:8], "sum": sum(v)}
        for name in ("commit_date", "receipt_date", "ship_mode", "o_priority", "c_nation", "p_type"):
            v = column(name, 64, seed, off)
            cols[name] = {"head": v[:8], "sum": sum(v)}
        cols["o_comment"] = {"head": column("o_comment", 4, seed, off)}
        out["generator"]["%d_%d" % (seed, off)] = cols
    for n, seed in ((3000, 42), (2500, 9)):
        li = {c: column(c, n, seed) for c in ("ship_date", "quantity", "ext_price", "discount", "tax", "flag",
                                              "status")}
        out["q6"]["%d_%d" % (n, seed)] = q6(li)
        out["q6"]["%d_%d_wide" % (n, seed)] = q6(li, 0, 2527, 0, 10, 51)
        out["q1"]["%d_%d" % (n, seed)] = q1(li)
        out["q1"]["%d_%d_cut100" % (n, seed)] = q1(li, 100)
    out["q3"]["300_1200_4800_42"] = q3(300, 1200, 4800, 42)
    out["q3"]["200_900_3000_5_seg3"] = q3(200, 900, 3000, 5, segment=3, date_lt=2000, ship_gt=300, k=20)
    out["q9"]["400_40_1500_6000_42"] = q9(400, 40, 1500, 6000, 42)
    out["q4"]["3000_12000_42"] = q4(3000, 12000, 42)
    out["q4"]["2000_9000_5_wide"] = q4(2000, 9000, 5, 0, 2406)
    out["q12"]["3000_12000_42"] = q12(3000, 12000, 42)
    out["q12"]["2000_9000_5_air_truck_hi3"] = q12(2000, 9000, 5, 0, 2600, (0, 6), 3)
    out["q13"]["300_3000_42"] = q13(300, 3000, 42)
    out["q10"]["300_3000_12000_42"] = q10(300, 3000, 12000, 42)
    out["q5"]["300_40_3000_12000_42"] = q5(300, 40, 3000, 12000, 42)
    out["q7"]["400_40_600_3000_12000_42"] = q7(400, 40, 600, 3000, 12000, 42)
    out["q7"]["400_40_600_3000_12000_5_peru_china_all"] = q7(400, 40, 600, 3000, 12000, 5, 17, 18, 0, 2556)
    out["q8"]["400_40_300_3000_12000_42_type7"] = q8(400, 40, 300, 3000, 12000, 42, 2, (1, 2, 3, 17, 24), 7)
    out["q8"]["500_40_300_4000_16000_9_japan_asia_1993_1997"] = q8(500, 40, 300, 4000, 16000, 9, 12,
                                                                   (8, 9, 12, 18, 21), 103, 366, 2191)
    out["q5"]["500_60_4000_16000_3_europe_all_years"] = q5(500, 60, 4000, 16000, 3, 0, 2406, (6, 7, 19, 22, 23))
    out["q10"]["200_2000_9000_5_wide"] = q10(200, 2000, 9000, 5, 0, 2406, 7)
    out["q13"]["200_4000_9_pinto_beans"] = q13(200, 4000, 9, "pinto", "beans")
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print(path)


if __name__ == "__main__":
    main()
