"""The multi-GPU form of the scans on CPU: world size 2 over gloo. Each rank generates its
row shard [rank*rows, (rank+1)*rows) of one seeded table with the engine's host generator
(bench.py's weak-scaling layout), computes its partial results (the oracle stands in for
the GPU here), and the partials travel as the engine's result structs; rank 0 merges them
with the engine's own merge functions (gpudb_q6_result_merge / gpudb_q1_result_merge), and
the merge must equal the result over the whole table. Also covers the max-over-ranks
timing reduction used by bench.py."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def q1_struct(capi, d):
    """gpudb_q1_result of a {(flag, status): sums} dict (groups in (flag, status) order)."""
    r = capi.Q1Result()
    for (f, st), v in sorted(d.items()):
        g = r.groups[r.n_groups]
        r.n_groups += 1
        g.flag, g.status, g.count = f, st, v["count"]
        for name in ("sum_qty", "sum_base_price", "sum_disc_price", "sum_charge", "sum_discount"):
            getattr(g, name).set(v[name])
    return r


def _worker(rank, world, port, rows, out):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    sys.path.insert(0, os.path.dirname(here))
    import ctypes as C

    import numpy as np
    import torch

    from gpudbmetalbenchmark_b200 import capi
    import oracle_py as orc

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    lib = capi.load()
    cols = {}
    for name, cid in (("ship_date", 1), ("quantity", 2), ("ext_price", 3), ("discount", 4), ("tax", 5),
                      ("flag", 6), ("status", 7)):
        spec = capi.GenSpec(seed=42, row_offset=rank * rows, n_rows=rows)
        a = np.empty(rows, dtype=orc.DT[lib.gpudb_column_width(cid)])
        assert lib.gpudb_generate(None, C.byref(spec), cid, a.ctypes.data, capi.MEM_HOST) == capi.OK
        cols[name] = a
    r6 = capi.Q6Result(*orc.q6(cols))
    r1 = q1_struct(capi, orc.q1(cols))
    gathered = [None] * world
    dist.all_gather_object(gathered, (bytes(r6), bytes(r1)))
    # the bench's timing reduction: max over ranks
    t = torch.tensor([float(rank + 1)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    if rank == 0:
        out.put((gathered, float(t.item())))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_shards_add_up_to_the_whole_table(orc):
    world, rows = 2, 60_000
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, rows, q)) for r in range(world)]
    for p in procs:
        p.start()
    gathered, tmax = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert tmax == 2.0
    from gpudbmetalbenchmark_b200 import capi
    from gpudbmetalbenchmark_b200.engine import q1_to_dict
    whole = orc.lineitem(world * rows, seed=42)
    p6 = [capi.Q6Result.from_buffer_copy(g[0]) for g in gathered]
    p1 = [capi.Q1Result.from_buffer_copy(g[1]) for g in gathered]
    m6 = capi.merge_q6(p6)
    assert (m6.revenue, m6.rows_matched) == orc.q6(whole)
    assert q1_to_dict(capi.merge_q1(p1)) == orc.q1(whole)
    assert q1_to_dict(capi.merge_q1(p1[::-1])) == orc.q1(whole)


def _leaving_worker(rank, world, port, out):
    import datetime
    import torch

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=5))
    t = torch.ones(1)
    dist.all_reduce(t)                      # step 1: both ranks
    if rank == 1:
        os._exit(0)                         # leaves between steps, with nothing in flight
    try:
        dist.all_reduce(t)                  # step 2: the peer is gone
        out.put("completed")
    except Exception as e:                  # noqa: BLE001 -- any error is the expected outcome
        out.put("error: " + type(e).__name__)


def test_a_rank_that_leaves_between_steps_fails_the_next_collective():
    """The survivor's next collective ends with an error inside the process-group timeout
    (5 s) instead of waiting for good."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_leaving_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    outcome = q.get(timeout=60)
    for p in procs:
        p.join(timeout=60)
    assert outcome.startswith("error"), outcome
