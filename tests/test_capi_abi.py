"""The C ABI without a GPU: the library loads, exports every function include/gpudb_capi.h
declares, generates tables on the host cores identically to the oracle's generator, and
fails cleanly (status codes, no crash) where a device would be needed."""
import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

from gpudbmetalbenchmark_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        names |= set(re.findall(r"\b(gpudb_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_every_declared_symbol_is_exported():
    lib = capi.load()
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the ctypes binding declares exactly the header's functions
    assert set(capi.PROTOTYPES) == set(names)


def test_abi_version_and_widths():
    lib = capi.load()
    assert lib.gpudb_abi_version() == 1
    for name, cid in capi.COL.items():
        w = lib.gpudb_column_width(cid)
        assert w in (1, 4, 8) or (name == "OR_COMMENT" and w == capi.COMMENT_WIDTH), name
    assert lib.gpudb_column_width(999) == 0


@pytest.mark.parametrize("col,kw", [(1, {}), (3, {}), (6, {}), (8, dict(n_orders=999, order_mode=1)),
                                    (8, dict(n_orders=999, order_mode=2)), (10, dict(n_parts=3000, n_supp=200)),
                                    (31, dict(n_cust=55)), (41, {}), (51, {}), (61, dict(n_supp=200)), (62, {}),
                                    (11, {}), (12, {}), (13, {}), (33, {}), (34, {}), (22, {}), (42, {})])
def test_host_generator_matches_oracle(orc, col, kw):
    lib = capi.load()
    n, off = 50_000, 777
    spec = capi.GenSpec(seed=9, row_offset=off, n_rows=n, n_orders=kw.get("n_orders", 0), n_cust=kw.get("n_cust", 0),
                        n_parts=kw.get("n_parts", 0), n_supp=kw.get("n_supp", 0), order_mode=kw.get("order_mode", 0))
    want = orc.gen(col, n, 9, off, **kw)
    got = np.empty_like(want)
    assert lib.gpudb_generate(None, C.byref(spec), col, got.ctypes.data, capi.MEM_HOST) == capi.OK
    assert np.array_equal(got, want)


def test_generator_rejects_bad_specs():
    lib = capi.load()
    buf = np.empty(10, np.int32)
    spec = capi.GenSpec(seed=1, n_rows=10)
    assert lib.gpudb_generate(None, C.byref(spec), 8, buf.ctypes.data, capi.MEM_HOST) == capi.E_INVALID  # no n_orders
    assert lib.gpudb_generate(None, C.byref(spec), 999, buf.ctypes.data, capi.MEM_HOST) == capi.E_INVALID
    assert lib.gpudb_generate(None, C.byref(spec), 1, buf.ctypes.data, capi.MEM_DEVICE) == capi.E_INVALID  # needs ctx


def test_null_context_is_rejected():
    lib = capi.load()
    li = capi.Lineitem()
    p6, r6 = capi.Q6Params(), capi.Q6Result()
    assert lib.gpudb_q6_sum(None, C.byref(li), C.byref(p6), C.byref(r6), None, None) == capi.E_INVALID
    assert lib.gpudb_sync(None) == capi.E_INVALID
    assert lib.gpudb_destroy(None) == capi.OK
    assert lib.gpudb_set_option(None, capi.OPT_CHUNK_ROWS, 1024) == capi.E_INVALID
    assert lib.gpudb_last_error_string(None) == b"no context"


def test_create_without_a_gpu_reports_no_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = capi.load()
    ctx = C.c_void_p()
    assert lib.gpudb_create(0, C.byref(ctx)) == capi.E_NODEVICE
    assert not ctx.value


def test_nation_region_and_part_type_helpers():
    """The host helpers behind the Q5/Q7/Q8 parameters: the TPC-H nation -> region table
    (five nations per region), region masks and p_type codes (GPUDB_PART_TYPE)."""
    assert sorted(capi.NATION_REGION.count(r) for r in range(5)) == [5] * 5
    assert capi.region_mask("ASIA") == (1 << 8) | (1 << 9) | (1 << 12) | (1 << 18) | (1 << 21)
    assert capi.region_mask(1) == (1 << 1) | (1 << 2) | (1 << 3) | (1 << 17) | (1 << 24)
    assert sum(capi.region_mask(r) for r in capi.REGION_NAMES) == (1 << 25) - 1
    assert capi.part_type("ECONOMY ANODIZED STEEL") == 103 == 4 * 25 + 0 * 5 + 3
    assert capi.part_type("STANDARD ANODIZED TIN") == 0 and capi.part_type("PROMO BRUSHED COPPER") == 149
    assert capi.NATION_NAMES.index("BRAZIL") == 2 and capi.NATION_NAMES.index("FRANCE") == 6
