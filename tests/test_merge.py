"""Shard merges of the C ABI (host-only, no GPU): Q9 groups of fact shards and Q3 top-k
lists of order-disjoint shards merge into the whole table's result, exactly; malformed
input is rejected. The per-shard results come from the oracle (these run on the CPU)."""
import pytest

from gpudbmetalbenchmark_b200 import capi
from gpudbmetalbenchmark_b200.engine import q3_to_list


def test_q9_groups_of_fact_shards_merge(orc):
    pa, su, ps, od, li = orc.q9_tables(4000, 300, 20_000, 120_000, 9)
    want, n_want = orc.q9(pa, su, ps, od, li)
    cuts = [0, 17_000, 60_001, 60_001, 120_000]   # one empty shard
    parts = []
    for a, b in zip(cuts, cuts[1:]):
        got, n = orc.q9(pa, su, ps, od, {k: v[a:b] for k, v in li.items()})
        assert n == len(got)
        parts.append(got)
    merged, n = capi.merge_q9(parts)
    assert (merged, n) == (want, n_want)
    # capacity below the group count: the total is still reported
    few, n2 = capi.merge_q9(parts, capacity=5)
    assert n2 == n_want and few == want[:5]


@pytest.mark.parametrize("k", [1, 10, 64])
def test_q3_top_k_of_order_disjoint_shards_merge(orc, k):
    cu, od, li = orc.q3_tables(3000, 30_000, 120_000, 5)
    want = orc.q3(cu, od, li, k=k)
    parts = []
    for shard in range(3):   # lineitem split by order key: each order's rows in one shard
        keep = (li["order_key"] // 4) % 3 == shard
        top, groups = orc.q3(cu, od, {c: v[keep] for c, v in li.items()}, k=k)
        r = capi.Q3Result()
        r.n_groups, r.n_rows = groups, len(top)
        for i, (key, date, rev) in enumerate(top):
            r.rows[i].order_key, r.rows[i].order_date, r.rows[i].revenue = key, date, rev
        parts.append(r)
    assert q3_to_list(capi.merge_q3(parts, k)) == want


def test_merges_reject_bad_input():
    bad = capi.Q1Result()
    bad.n_groups = 1
    bad.groups[0].flag = 7
    with pytest.raises(capi.GpudbError):
        capi.merge_q1([bad])
    with pytest.raises(capi.GpudbError):
        capi.merge_q3([capi.Q3Result()], 0)
    assert capi.merge_q6([]).rows_matched == 0
    assert capi.merge_q9([]) == ([], 0)
