"""Failure paths, made without a GPU fault: a device wait that nothing completes gives up
after its bound and reports GPUDB_E_TIMEOUT; an allocation the device cannot satisfy
reports GPUDB_E_OOM; a serving wait with no time left reports GPUDB_E_TIMEOUT and the
request still completes; bad arguments report GPUDB_E_INVALID. After each, the same
context keeps producing exact results."""
import ctypes as C
import time

import pytest

from gpudbmetalbenchmark_b200 import capi
from gpudbmetalbenchmark_b200.engine import Engine

pytestmark = pytest.mark.gpu


def still_exact(e, orc, li, t):
    assert e.q6(t, 100, 900, 2, 8, 30) == orc.q6(li, 100, 900, 2, 8, 30)


def test_bounded_device_wait_times_out(orc):
    li = orc.lineitem(50_000, seed=31)
    with Engine(0) as e:
        t = e.upload("lineitem", li)
        assert e.lib.gpudb_selftest_bounded_wait(e.ctx, 4096, 1) == capi.OK      # the barrier completes
        t0 = time.perf_counter()
        rc = e.lib.gpudb_selftest_bounded_wait(e.ctx, 4096, 0)                  # nothing ever arrives
        assert rc == capi.E_TIMEOUT and time.perf_counter() - t0 < 3.0
        assert b"bounded device wait" in e.lib.gpudb_last_error_string(e.ctx)
        still_exact(e, orc, li, t)
        assert e.lib.gpudb_selftest_bounded_wait(e.ctx, 0, 0) == capi.E_INVALID


def test_device_allocation_failure(orc):
    li = orc.lineitem(20_000, seed=32)
    with Engine(0) as e:
        t = e.upload("lineitem", li)
        p = C.c_void_p()
        assert e.lib.gpudb_device_alloc(e.ctx, 1 << 50, C.byref(p)) == capi.E_OOM
        still_exact(e, orc, li, t)


def test_serving_wait_with_no_time_left(engine):
    from gpudbmetalbenchmark_b200.serve import Server
    t = engine.generate("lineitem", 60_000_000, seed=42, columns=("ship_date", "quantity", "ext_price", "discount",
                                                                 "tax", "flag", "status"))
    s = t.lineitem()
    r = capi.Request(pipeline=capi.PIPE_Q1)
    r.li = C.pointer(s)
    r.q1 = capi.Q1Params(2436, 0)
    out = capi.Q1Result()
    r.q1_out = C.pointer(out)
    srv = Server(lanes=1, max_batch=1)
    try:
        ticket = srv.submit(r)
        rc, _ = srv.wait(ticket, timeout_ms=0.0)
        assert rc == capi.E_TIMEOUT                 # still queued or running
        rc, lat = srv.wait(ticket, timeout_ms=60000.0)
        assert rc == capi.OK and lat > 0 and out.n_groups == 6
    finally:
        srv.close()
        engine.free(t)


def test_bad_arguments(engine):
    assert engine.lib.gpudb_set_option(engine.ctx, capi.OPT_HT_LOAD, 40) == capi.E_INVALID
    assert engine.lib.gpudb_set_option(engine.ctx, 999, 1) == capi.E_INVALID
    assert engine.lib.gpudb_q6_sum(engine.ctx, None, None, None, None, None) == capi.E_INVALID
    cfg = capi.ServeConfig(device=0, lanes=0, max_batch=1)
    h = C.c_void_p()
    assert engine.lib.gpudb_serve_open(C.byref(cfg), C.byref(h)) == capi.E_INVALID
