"""gpudb_q6_sum_noalloc: the filtered sum for callers that cannot allocate device memory
(device memory owned and budgeted by another memory manager, or no gpudb context). Its
result must equal the allocating entry point gpudb_q6_sum exactly, on consecutive calls
that share the static scratch array. This file sorts last so that a failure here comes
after every other test has run."""
import ctypes as C

import numpy as np
import pytest

from gpudbmetalbenchmark_b200 import Engine, capi

pytestmark = pytest.mark.gpu


def _noalloc(eng, li_struct, params, out, stream):
    return eng.lib.gpudb_q6_sum_noalloc(C.byref(li_struct), C.byref(params), out, stream)


def test_noalloc_matches_allocating_entry_point(orc):
    with Engine(0) as eng:
        n = 1_000_003
        li = orc.lineitem(n, seed=31)
        t = eng.upload("lineitem", li)
        out = eng.device_array(16)
        stream = eng.lib.gpudb_stream(eng.ctx)   # order the call with the copies below
        cases = [(365, 730, 5, 7, 24), (0, 2527, 0, 10, 51), (365, 730, 5, 7, 24), (1000, 1200, 3, 4, 30)]
        for view, sub in ((t.lineitem(), li), (t.lineitem(n_rows=n - 3, row_offset=3), {k: v[3:] for k, v in li.items()})):
            for lo, hi, dlo, dhi, qlt in cases:     # consecutive calls share the scratch array
                p = capi.Q6Params(lo, hi, dlo, dhi, qlt)
                assert _noalloc(eng, view, p, out, stream) == capi.OK
                got = tuple(int(x) for x in eng.to_host(out, 2, np.int64))
                want = eng.q6(view, lo, hi, dlo, dhi, qlt)
                assert got == want
                assert got == orc.q6(sub, lo, hi, dlo, dhi, qlt)
        eng.device_free(out)


def test_noalloc_at_its_row_limit():
    """Exactly 67,108,864 rows: every block of the largest grid writes its partial and the
    last one folds them all; two calls in a row agree with the allocating entry point."""
    from gpudbmetalbenchmark_b200.engine import Q6_COLS
    n = 67_108_864
    with Engine(0) as eng:
        t = eng.generate("lineitem", n, seed=5, columns=Q6_COLS)
        out = eng.device_array(16)
        stream = eng.lib.gpudb_stream(eng.ctx)
        for lo, hi, dlo, dhi, qlt in ((365, 730, 5, 7, 24), (0, 2527, 0, 10, 51)):
            p = capi.Q6Params(lo, hi, dlo, dhi, qlt)
            assert _noalloc(eng, t.lineitem(), p, out, stream) == capi.OK
            got = tuple(int(x) for x in eng.to_host(out, 2, np.int64))
            assert got == eng.q6(t, lo, hi, dlo, dhi, qlt)
        eng.device_free(out)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    with Engine(0) as eng:
        li = capi.Lineitem()
        li.location = capi.MEM_DEVICE
        li.n_rows = 67_108_864 + 1
        buf = eng.device_array(64)
        li.ship_date = li.discount = li.quantity = li.ext_price = buf
        p = capi.Q6Params(365, 730, 5, 7, 24)
        assert _noalloc(eng, li, p, buf, None) == capi.E_CAPACITY
        li.location = capi.MEM_HOST
        assert _noalloc(eng, li, p, buf, None) == capi.E_INVALID
        eng.device_free(buf)
