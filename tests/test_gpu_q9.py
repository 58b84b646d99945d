"""Q9-like star join + (nation, year) aggregate on the GPU against the CPU oracle, bit-exact:
the full config 3 sizes, small tables, the shared-memory spill path, global-table overflow
reporting, a streamed fact table with ragged chunks and truncated outputs."""
import numpy as np
import pytest

from gpudbmetalbenchmark_b200 import capi

pytestmark = pytest.mark.gpu


def upload_all(engine, tabs, location=capi.MEM_DEVICE):
    pa, su, ps, od, li = tabs
    return [engine.upload("part", pa), engine.upload("supplier", su), engine.upload("partsupp", ps),
            engine.upload("orders", od), engine.upload("lineitem", li, location=location)]


def free_all(engine, ts):
    for t in ts:
        engine.free(t)


@pytest.mark.parametrize("sizes,seed", [((2_000_000, 100_000, 15_000_000, 60_000_000), 42),
                                        ((20_000, 1_000, 100_000, 500_000), 3), ((40, 8, 30, 100), 4)])
def test_q9_matches_oracle(engine, orc, sizes, seed):
    tabs = orc.q9_tables(*sizes, seed)
    ts = upload_all(engine, tabs)
    try:
        assert engine.q9(*ts) == orc.q9(*tabs)
    finally:
        free_all(engine, ts)


def test_q9_shared_table_spill_and_small_global_table(engine, orc):
    tabs = orc.q9_tables(20_000, 1_000, 100_000, 400_000, 8)
    ts = upload_all(engine, tabs)
    try:
        want = orc.q9(*tabs)
        assert want[1] > 100
        assert engine.q9(*ts, smem_slots=32) == want        # most groups spill to the global table
        assert engine.q9(*ts, global_slots=256) == want
        with pytest.raises(capi.GpudbError) as e:
            engine.q9(*ts, global_slots=64)                  # fewer slots than groups
        assert e.value.code == capi.E_CAPACITY
        with pytest.raises(capi.GpudbError) as e:
            engine.q9(*ts, smem_slots=100)                   # not a power of two
        assert e.value.code == capi.E_INVALID
        rows, n = engine.q9(*ts, capacity=10)
        assert n == want[1] and rows == want[0][:10]
    finally:
        free_all(engine, ts)


@pytest.mark.parametrize("n_parts", [1_700_000, 3_300_000])
def test_q9_part_filter_past_shared_memory(engine, orc, n_parts):
    """Part keys past the shared-memory filter's 1,638,400 bits: a blocked Bloom filter in
    shared memory whose false positives the resolve drops after testing the exact bitmap."""
    tabs = orc.q9_tables(n_parts, 2_000, 200_000, 800_000, 17)
    ts = upload_all(engine, tabs)
    try:
        assert engine.q9(*ts) == orc.q9(*tabs)
    finally:
        free_all(engine, ts)


@pytest.mark.parametrize("piece", [0, 65_537])
def test_q9_fact_part_keys_outside_the_part_range(engine, orc, piece):
    """Fact rows whose part key is negative or above the part table's largest key match no
    part. In the Bloom form (more parts than the shared-memory bitmap holds) the filter does
    not test the range; such a key that passes the Bloom filter is turned away by the
    resolve before it reads the exact bitmap."""
    tabs = orc.q9_tables(1_700_000, 2_000, 200_000, 800_003, 23)
    li = tabs[4]
    part_max = int(tabs[0]["part_key"].max())
    rng = np.random.default_rng(5)
    rows = rng.choice(len(li["part_key"]), 40_000, replace=False)
    bad = np.array([-7, -1, part_max + 1, part_max + 1_000_003, 2**31 - 1, -2**31], np.int32)
    li["part_key"][rows] = bad[np.arange(len(rows)) % len(bad)]
    ts = upload_all(engine, tabs)
    try:
        kw = {"chunk_rows": piece} if piece else {}
        assert engine.q9(*ts, **kw) == orc.q9(*tabs)
    finally:
        free_all(engine, ts)


@pytest.mark.parametrize("piece", [40_000, 30_001])
def test_q9_fact_table_in_pieces(engine, orc, piece):
    """A device-resident fact table goes through the filter + resolve kernels in pieces of
    chunk_rows rows (an odd size starts pieces off the 16-byte boundary: scalar loads)."""
    tabs = orc.q9_tables(20_000, 1_000, 100_000, 300_001, 13)
    ts = upload_all(engine, tabs)
    try:
        assert engine.q9(*ts, chunk_rows=piece) == orc.q9(*tabs)
    finally:
        free_all(engine, ts)


def test_q9_streamed_fact_table(engine, orc):
    tabs = orc.q9_tables(20_000, 1_000, 100_000, 300_001, 9)
    ts = upload_all(engine, tabs, location=capi.MEM_HOST)
    try:
        assert engine.q9(*ts, chunk_rows=40_000) == orc.q9(*tabs)
    finally:
        free_all(engine, ts)


def test_q9_no_flagged_part(engine, orc):
    tabs = orc.q9_tables(2_000, 100, 3_000, 10_000, 5)
    tabs[0]["flag"][:] = 0
    ts = upload_all(engine, tabs)
    try:
        assert engine.q9(*ts) == ([], 0)
    finally:
        free_all(engine, ts)


def test_q9_key_out_of_range_reported(engine, orc):
    tabs = orc.q9_tables(2_000, 100, 3_000, 10_000, 5)
    ts = upload_all(engine, tabs)
    try:
        s = ts[1].struct()
        s.key_max = 50   # suppliers 51..99 fall outside the declared range
        import ctypes as C
        groups = (capi.Q9Group * 64)()
        n = C.c_uint32()
        rc = engine.lib.gpudb_q9_star(engine.ctx, C.byref(ts[0].struct()), C.byref(s), C.byref(ts[2].struct()),
                                      C.byref(ts[3].struct()), C.byref(ts[4].lineitem()), None, groups, 64,
                                      C.byref(n), None, None)
        assert rc == capi.E_KEY_RANGE
    finally:
        free_all(engine, ts)


def test_q9_graph_capture_and_replay(orc):
    """A device-resident Q9 call is captured into a CUDA graph once and replayed: the first
    (capturing) call, replays, a changed parameter (a new capture) and graphs switched off all
    give the oracle's groups; replays count the graph's kernels as launches."""
    from gpudbmetalbenchmark_b200.engine import Engine
    tabs = orc.q9_tables(20_000, 1_000, 100_000, 400_000, 11)
    want = orc.q9(*tabs)
    with Engine(0) as e:
        assert e.get_option(capi.OPT_GRAPHS) == 1
        ts = upload_all(e, tabs)
        kernels = []
        for _ in range(3):
            t = capi.Timing()
            assert e.q9(*ts, timing=t) == want
            kernels.append(t.kernels)
        assert kernels[0] == kernels[1] == kernels[2] == 9
        before = e.launches()
        assert e.q9(*ts, smem_slots=64) == want          # another key: captured anew
        assert e.q9(*ts, smem_slots=64) == want
        assert e.launches() - before == 18
        with pytest.raises(capi.GpudbError) as err:       # device status still reported from a graph
            e.q9(*ts, global_slots=64)
        assert err.value.code == capi.E_CAPACITY
        e.set_option(capi.OPT_GRAPHS, 0)
        assert e.q9(*ts) == want
        e.set_option(capi.OPT_GRAPHS, 1)
        assert e.q9(*ts) == want
