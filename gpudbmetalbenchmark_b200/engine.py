"""Host-side mirror of the reference's per-pipeline operator surface, over the C ABI.

The reference exposes one entry per pipeline, `runQnBenchmark(device, queue, library)`
(src/infra.h:874-922), that loads its tables, runs the kernels and prints the result. Here
`Engine` owns a context (device + streams, the analogue of the device/queue/library
triple), `Table` objects own HBM-resident (or pinned host) columns, and one method per
pipeline returns the exact result as Python integers. Every method calls the CUDA
library; a missing library or GPU is an error, never a CPU fallback.
"""
import ctypes as C
import os

import numpy as np

from . import capi
from .capi import COL, MEM_DEVICE, MEM_HOST

DTYPES = {1: np.uint8, 4: np.int32, 8: np.int64, capi.COMMENT_WIDTH: np.dtype("S%d" % capi.COMMENT_WIDTH)}

LINEITEM_COLS = {  # field of capi.Lineitem -> column id
    "ship_date": COL["LI_SHIP_DATE"], "quantity": COL["LI_QUANTITY"], "ext_price": COL["LI_EXT_PRICE"],
    "discount": COL["LI_DISCOUNT"], "tax": COL["LI_TAX"], "flag": COL["LI_FLAG"], "status": COL["LI_STATUS"],
    "order_key": COL["LI_ORDER_KEY"], "part_key": COL["LI_PART_KEY"], "supp_key": COL["LI_SUPP_KEY"],
    "commit_date": COL["LI_COMMIT_DATE"], "receipt_date": COL["LI_RECEIPT_DATE"], "ship_mode": COL["LI_SHIP_MODE"],
}
Q4_LI_COLS = ("order_key", "commit_date", "receipt_date")
Q12_LI_COLS = ("order_key", "ship_date", "commit_date", "receipt_date", "ship_mode")
Q1_COLS = ("ship_date", "quantity", "ext_price", "discount", "tax", "flag", "status")
Q6_COLS = ("ship_date", "discount", "quantity", "ext_price")
TABLE_COLS = {
    "customer": {"cust_key": COL["CU_CUST_KEY"], "segment": COL["CU_SEGMENT"], "nation": COL["CU_NATION"]},
    "orders": {"order_key": COL["OR_ORDER_KEY"], "cust_key": COL["OR_CUST_KEY"], "order_date": COL["OR_ORDER_DATE"],
               "priority": COL["OR_PRIORITY"], "comment": COL["OR_COMMENT"]},
    "part": {"part_key": COL["PA_PART_KEY"], "flag": COL["PA_FLAG"], "type": COL["PA_TYPE"]},
    "supplier": {"supp_key": COL["SU_SUPP_KEY"], "nation": COL["SU_NATION"]},
    "partsupp": {"part_key": COL["PS_PART_KEY"], "supp_key": COL["PS_SUPP_KEY"], "supply_cost": COL["PS_SUPPLY_COST"]},
    "lineitem": LINEITEM_COLS,
}


class Table:
    """Columns of one table in device memory (or pinned host memory) owned by the engine."""

    def __init__(self, engine, kind, n_rows, location, key_max=None):
        self.engine, self.kind, self.n_rows, self.location = engine, kind, n_rows, location
        self.cols = {}          # name -> (pointer, column id)
        self.key_max = dict(key_max or {})

    def ptr(self, name):
        return self.cols[name][0] if name in self.cols else None

    def to_numpy(self, name):
        ptr, cid = self.cols[name]
        w = capi.load().gpudb_column_width(cid)
        out = np.empty(self.n_rows, dtype=DTYPES[w])
        if self.n_rows:
            self.engine._check(capi.load().gpudb_copy(self.engine.ctx, out.ctypes.data, ptr, self.n_rows * w))
        return out

    def host_view(self, name):
        """Zero-copy numpy view of a pinned host column."""
        assert self.location == MEM_HOST
        ptr, cid = self.cols[name]
        w = capi.load().gpudb_column_width(cid)
        buf = (C.c_uint8 * (self.n_rows * w)).from_address(ptr)
        return np.frombuffer(buf, dtype=DTYPES[w])

    def close(self):
        lib = capi.load()
        for ptr, _ in self.cols.values():
            if ptr:
                if self.location == MEM_DEVICE:
                    lib.gpudb_device_free(self.engine.ctx, ptr)
                else:
                    lib.gpudb_host_free(self.engine.ctx, ptr)
        self.cols = {}

    # ---- C structs -------------------------------------------------------------------
    def lineitem(self, n_rows=None, row_offset=0):
        li = capi.Lineitem()
        li.n_rows = self.n_rows if n_rows is None else n_rows
        li.location = self.location
        li.order_key_max = self.key_max.get("order_key", -1)
        for name, (ptr, cid) in self.cols.items():
            w = capi.load().gpudb_column_width(cid)
            setattr(li, name, ptr + row_offset * w if ptr else None)
        return li

    def struct(self):
        if self.kind == "lineitem":
            return self.lineitem()
        cls = {"customer": capi.Customer, "orders": capi.Orders, "part": capi.Part,
               "supplier": capi.Supplier, "partsupp": capi.Partsupp}[self.kind]
        s = cls()
        s.n_rows = self.n_rows
        for name, (ptr, _) in self.cols.items():
            setattr(s, name, ptr)
        if self.kind == "orders":
            s.key_max = self.key_max.get("order_key", -1)
            s.cust_key_max = self.key_max.get("cust_key", -1)
        elif self.kind in ("customer", "part", "supplier"):
            s.key_max = self.key_max.get("key", -1)
        return s


class Engine:
    def __init__(self, device=0):
        self.lib = capi.load()
        ctx = C.c_void_p()
        rc = self.lib.gpudb_create(device, C.byref(ctx))
        if rc != capi.OK:
            raise capi.GpudbError(rc, "gpudb_create(%d) failed" % device)
        self.ctx = ctx
        self.tables = []

    def close(self):
        if self.ctx:
            for t in self.tables:
                t.close()
            self.tables = []
            self.lib.gpudb_destroy(self.ctx)
            self.ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc):
        if rc != capi.OK:
            raise capi.GpudbError(rc, self.lib.gpudb_last_error_string(self.ctx).decode())
        return rc

    def launches(self):
        return self.lib.gpudb_kernel_launches(self.ctx)

    def set_chunk_rows(self, rows):
        """Rows per streamed chunk when a lineitem table lives in host memory."""
        return self._check(self.lib.gpudb_set_option(self.ctx, capi.OPT_CHUNK_ROWS, int(rows)))

    def set_scan_variant(self, variant):
        """Q1 scan kernel choice (GPUDB_OPT_SCAN_VARIANT): 0 auto, 1..7 (see gpudb_capi.h)."""
        return self._check(self.lib.gpudb_set_option(self.ctx, capi.OPT_SCAN_VARIANT, int(variant)))

    def set_option(self, option, value):
        return self._check(self.lib.gpudb_set_option(self.ctx, int(option), int(value)))

    def get_option(self, option):
        v = C.c_int64()
        self._check(self.lib.gpudb_get_option(self.ctx, int(option), C.byref(v)))
        return v.value

    def autotune(self, req, reps=10):
        """Times the candidate settings of one request's pipeline (a capi.Request) on its own
        tables and keeps the fastest on this context; returns what was chosen."""
        r = capi.TuneResult()
        self._check(self.lib.gpudb_autotune(self.ctx, C.byref(req), int(reps), C.byref(r)))
        out = {"pipeline": r.pipeline, "candidates": r.candidates, "dropped": r.dropped,
               capi.OPT_NAMES[r.option]: r.value, "best_ms": r.best_ms, "default_ms": r.default_ms}
        if r.option2:
            out[capi.OPT_NAMES[r.option2]] = r.value2
        return out

    def tune_save(self, path):
        return self._check(self.lib.gpudb_tune_save(self.ctx, os.fsencode(path)))

    def tune_load(self, path):
        n = C.c_uint32()
        self._check(self.lib.gpudb_tune_load(self.ctx, os.fsencode(path), C.byref(n)))
        return n.value

    def sync(self):
        return self._check(self.lib.gpudb_sync(self.ctx))

    # ---- tables ------------------------------------------------------------------------
    def _alloc(self, nbytes, location):
        p = C.c_void_p()
        fn = self.lib.gpudb_device_alloc if location == MEM_DEVICE else self.lib.gpudb_host_alloc
        self._check(fn(self.ctx, max(nbytes, 1), C.byref(p)))
        return p.value

    def generate(self, kind, n_rows, seed=42, columns=None, location=MEM_DEVICE, row_offset=0,
                 n_orders=0, n_cust=0, n_parts=0, n_supp=0, order_mode=capi.ORDERS_NONE):
        """Generate a synthetic table (device kernels for MEM_DEVICE, host cores for MEM_HOST)."""
        spec = capi.GenSpec(seed=seed, row_offset=row_offset, n_rows=n_rows, n_orders=n_orders, n_cust=n_cust,
                            n_parts=n_parts, n_supp=n_supp, order_mode=order_mode)
        names = list(columns) if columns is not None else list(TABLE_COLS[kind])
        t = Table(self, kind, n_rows, location)
        for name in names:
            cid = TABLE_COLS[kind][name]
            w = self.lib.gpudb_column_width(cid)
            ptr = self._alloc(n_rows * w, location)
            t.cols[name] = (ptr, cid)
            self._check(self.lib.gpudb_generate(self.ctx, C.byref(spec), cid, ptr, location))
        last = row_offset + n_rows - 1
        if kind == "lineitem" and "order_key" in t.cols:
            t.key_max["order_key"] = 4 * (n_orders - 1) + 1
        elif kind == "orders":
            t.key_max["order_key"] = 4 * last + 1
            t.key_max["cust_key"] = n_cust - 1
        elif kind in ("customer", "part", "supplier"):
            t.key_max["key"] = last
        self.tables.append(t)
        return t

    def upload(self, kind, arrays, key_max=None, location=MEM_DEVICE):
        """Copy numpy columns into a new table."""
        n = len(next(iter(arrays.values())))
        t = Table(self, kind, n, location, key_max)
        for name, arr in arrays.items():
            cid = TABLE_COLS[kind][name]
            w = self.lib.gpudb_column_width(cid)
            a = np.ascontiguousarray(arr, dtype=DTYPES[w])
            assert len(a) == n
            ptr = self._alloc(n * w, location)
            t.cols[name] = (ptr, cid)
            if n:
                self._check(self.lib.gpudb_copy(self.ctx, ptr, a.ctypes.data, n * w))
        if key_max is None:
            if kind == "lineitem" and "order_key" in arrays:
                t.key_max["order_key"] = int(arrays["order_key"].max()) if n else -1
            elif kind == "orders":
                if "order_key" in arrays:
                    t.key_max["order_key"] = int(arrays["order_key"].max()) if n else -1
                if "cust_key" in arrays:
                    t.key_max["cust_key"] = int(arrays["cust_key"].max()) if n else -1
            elif kind in ("customer", "part", "supplier"):
                k = {"customer": "cust_key", "part": "part_key", "supplier": "supp_key"}[kind]
                t.key_max["key"] = int(arrays[k].max()) if n else -1
        self.tables.append(t)
        return t

    def load_tbl(self, kind, source, columns=None, timing=None):
        """Parse dbgen-style '|'-separated text (a path, or bytes) on the GPU into a new
        device table of `kind` (gpudb_tbl_parse); `columns` limits the columns kept."""
        data = source if isinstance(source, (bytes, bytearray)) else open(source, "rb").read()
        buf = np.frombuffer(data, dtype=np.uint8) if len(data) else np.zeros(1, np.uint8)
        code, names = capi.TBL_COLUMNS[kind]
        n = C.c_uint64()
        self._check(self.lib.gpudb_tbl_count_rows(self.ctx, buf.ctypes.data, len(data), MEM_HOST, C.byref(n)))
        t = Table(self, kind, n.value, MEM_DEVICE)
        cols = (C.c_void_p * capi.TBL_MAX_COLS)()
        for i, name in enumerate(names):
            if columns is not None and name not in columns:
                continue
            cid = TABLE_COLS[kind][name]
            ptr = self._alloc(n.value * self.lib.gpudb_column_width(cid), MEM_DEVICE)
            t.cols[name] = (ptr, cid)
            cols[i] = ptr
        self.tables.append(t)
        got = C.c_uint64()
        col_max = (C.c_int32 * capi.TBL_MAX_COLS)()
        self._check(self.lib.gpudb_tbl_parse(self.ctx, code, buf.ctypes.data, len(data), MEM_HOST, cols, n.value,
                                             C.byref(got), col_max, C.byref(timing) if timing is not None else None))
        assert got.value == n.value
        if kind == "lineitem":
            t.key_max["order_key"] = col_max[0] if n.value else -1
        elif kind == "orders":
            t.key_max["order_key"] = col_max[0] if n.value else -1
            t.key_max["cust_key"] = col_max[1] if n.value else -1
        elif kind in ("customer", "part", "supplier"):
            t.key_max["key"] = col_max[0] if n.value else -1
        return t

    def free(self, table):
        table.close()
        if table in self.tables:
            self.tables.remove(table)

    # ---- pipelines -----------------------------------------------------------------------
    @staticmethod
    def _exec(async_, stream):
        if not async_ and stream is None:
            return None
        return C.byref(capi.Exec(async_=1 if async_ else 0, flags=0, stream=stream))

    def q6(self, li, ship_lo=365, ship_hi=730, disc_lo=5, disc_hi=7, qty_lt=24, timing=None, async_=False,
           stream=None, out=None):
        """Filtered sum: (revenue in hundredths^2, rows matched)."""
        s = li if isinstance(li, capi.Lineitem) else li.lineitem()
        p = capi.Q6Params(ship_lo, ship_hi, disc_lo, disc_hi, qty_lt)
        r = out if out is not None else capi.Q6Result()
        self._check(self.lib.gpudb_q6_sum(self.ctx, C.byref(s), C.byref(p), C.byref(r),
                                          C.byref(timing) if timing is not None else None,
                                          self._exec(async_, stream)))
        return r if async_ else (r.revenue, r.rows_matched)

    def q1(self, li, ship_le=2436, timing=None, async_=False, stream=None, out=None):
        """6-group aggregate: {(flag, status): dict(count, sum_qty, ...)}."""
        s = li if isinstance(li, capi.Lineitem) else li.lineitem()
        p = capi.Q1Params(ship_le, 0)
        r = out if out is not None else capi.Q1Result()
        self._check(self.lib.gpudb_q1_group6(self.ctx, C.byref(s), C.byref(p), C.byref(r),
                                             C.byref(timing) if timing is not None else None,
                                             self._exec(async_, stream)))
        return r if async_ else q1_to_dict(r)

    def q3(self, cu, od, li, segment=1, order_date_lt=1170, ship_date_gt=1170, k=10, join_mode=capi.JOIN_GLOBAL,
           radix_bits=0, timing=None, async_=False, out=None):
        """Top-k (order_key, order_date, revenue) and the number of groups."""
        p = capi.Q3Params(segment, order_date_lt, ship_date_gt, k, join_mode, radix_bits)
        r = out if out is not None else capi.Q3Result()
        cs, os_, ls = cu.struct(), od.struct(), (li if isinstance(li, capi.Lineitem) else li.lineitem())
        self._check(self.lib.gpudb_q3_join_topk(self.ctx, C.byref(cs), C.byref(os_), C.byref(ls), C.byref(p),
                                                C.byref(r), C.byref(timing) if timing is not None else None,
                                                self._exec(async_, None)))
        return r if async_ else q3_to_list(r)

    def q4(self, od, li, date_lo=547, date_hi=639, timing=None, async_=False, out=None):
        """Orders per priority 1..5 in [date_lo, date_hi) with a late lineitem (commit < receipt).
        The defaults are the query's 1993-07-01 .. 1993-10-01 as day numbers."""
        p = capi.Q4Params(date_lo, date_hi)
        r = out if out is not None else capi.Q4Result()
        ls = li if isinstance(li, capi.Lineitem) else li.lineitem()
        self._check(self.lib.gpudb_q4_priority(self.ctx, C.byref(od.struct()), C.byref(ls), C.byref(p), C.byref(r),
                                               C.byref(timing) if timing is not None else None,
                                               self._exec(async_, None)))
        return r if async_ else list(r.count)

    def q12(self, od, li, receipt_lo=731, receipt_hi=1096, modes=(capi.MODE_MAIL, capi.MODE_SHIP), high_max=2,
            timing=None, async_=False, out=None):
        """[(high, low) for each of the two ship modes]: lineitem rows of that mode received in
        [receipt_lo, receipt_hi) (default: 1994) with ship < commit < receipt, split by order
        priority 1..high_max (high) or other (low)."""
        p = capi.Q12Params(receipt_lo, receipt_hi, (C.c_int32 * 2)(*modes), high_max, 0)
        r = out if out is not None else capi.Q12Result()
        ls = li if isinstance(li, capi.Lineitem) else li.lineitem()
        self._check(self.lib.gpudb_q12_shipmode(self.ctx, C.byref(od.struct()), C.byref(ls), C.byref(p), C.byref(r),
                                                C.byref(timing) if timing is not None else None,
                                                self._exec(async_, None)))
        return r if async_ else [(r.high[0], r.low[0]), (r.high[1], r.low[1])]

    def q5(self, cu, su, od, li, date_lo=731, date_hi=1096, region="ASIA", timing=None):
        """[(nation, revenue)] for the nations of `region` with revenue, ordered by revenue desc
        (then nation asc): lineitems of orders in [date_lo, date_hi) (default 1994) whose
        customer and supplier share the nation; revenue in hundredths^2."""
        p = capi.Q5Params(date_lo, date_hi, capi.region_mask(region), 0)
        r = capi.Q5Result()
        ls = li if isinstance(li, capi.Lineitem) else li.lineitem()
        self._check(self.lib.gpudb_q5_local_supplier(self.ctx, C.byref(cu.struct()), C.byref(su.struct()),
                                                     C.byref(od.struct()), C.byref(ls), C.byref(p), C.byref(r),
                                                     C.byref(timing) if timing is not None else None, None))
        return sorted(((n, r.revenue[n]) for n in range(capi.NATIONS) if r.revenue[n]), key=lambda x: (-x[1], x[0]))

    def q7(self, cu, su, od, li, nation_a="FRANCE", nation_b="GERMANY", ship_lo=1096, ship_hi=1826, timing=None):
        """[(supp_nation, cust_nation, year, revenue)] ordered by the nations' names, then year:
        lineitems shipped in [ship_lo, ship_hi] (default 1995-01-01 .. 1996-12-31) from a supplier
        of one nation to a customer of the other; revenue in hundredths^2."""
        na = capi.NATION_NAMES.index(nation_a) if isinstance(nation_a, str) else nation_a
        nb = capi.NATION_NAMES.index(nation_b) if isinstance(nation_b, str) else nation_b
        p = capi.Q7Params(na, nb, ship_lo, ship_hi)
        r = capi.Q7Result()
        ls = li if isinstance(li, capi.Lineitem) else li.lineitem()
        self._check(self.lib.gpudb_q7_volume_shipping(self.ctx, C.byref(cu.struct()), C.byref(su.struct()),
                                                      C.byref(od.struct()), C.byref(ls), C.byref(p), C.byref(r),
                                                      C.byref(timing) if timing is not None else None, None))
        rows = [(s, c, r.first_year + y, r.revenue[pair][y]) for pair, (s, c) in enumerate(((na, nb), (nb, na)))
                for y in range(r.n_years) if r.revenue[pair][y]]
        return sorted(rows, key=lambda x: (capi.NATION_NAMES[x[0]], capi.NATION_NAMES[x[1]], x[2]))

    def q8(self, cu, su, pa, od, li, nation="BRAZIL", region="AMERICA", part_type="ECONOMY ANODIZED STEEL",
           date_lo=1096, date_hi=1826, timing=None):
        """[(year, nation_volume, volume)] per calendar year of [date_lo, date_hi] (default 1995 and
        1996): revenue of the part type's lineitems whose order's customer is in the region, and
        the part supplied by the nation; the market share is nation_volume / volume."""
        n = capi.NATION_NAMES.index(nation) if isinstance(nation, str) else nation
        t = capi.part_type(part_type) if isinstance(part_type, str) else part_type
        p = capi.Q8Params(date_lo, date_hi, capi.region_mask(region), n, t, 0)
        r = capi.Q8Result()
        ls = li if isinstance(li, capi.Lineitem) else li.lineitem()
        self._check(self.lib.gpudb_q8_market_share(self.ctx, C.byref(cu.struct()), C.byref(su.struct()),
                                                   C.byref(pa.struct()), C.byref(od.struct()), C.byref(ls), C.byref(p),
                                                   C.byref(r), C.byref(timing) if timing is not None else None, None))
        return [(r.first_year + y, r.nation_volume[y], r.volume[y]) for y in range(r.n_years)]

    def q10(self, cu, od, li, date_lo=639, date_hi=731, k=20, timing=None):
        """([(cust_key, revenue)] top k by revenue desc, key asc; customers with revenue > 0):
        revenue of returned lineitems (flag 2, 'R') of orders in [date_lo, date_hi) per
        customer (default 1993-10-01 .. 1994-01-01), hundredths^2."""
        p = capi.Q10Params(date_lo, date_hi, k, 0)
        r = capi.Q10Result()
        ls = li if isinstance(li, capi.Lineitem) else li.lineitem()
        self._check(self.lib.gpudb_q10_returned(self.ctx, C.byref(cu.struct()), C.byref(od.struct()), C.byref(ls),
                                                C.byref(p), C.byref(r),
                                                C.byref(timing) if timing is not None else None, None))
        return [(x.cust_key, x.revenue) for x in r.rows[:r.n_rows]], r.n_customers

    def q13(self, cu, od, word1=b"special", word2=b"requests", capacity=capi.Q13_MAX_COUNT + 1, timing=None):
        """[(c_count, custdist)] ordered by custdist desc, c_count desc: customers per number of
        their orders whose comment is NOT LIKE '%word1%word2%'."""
        p = capi.Q13Params(word1, word2)
        rows = (capi.Q13Row * capacity)()
        n = C.c_uint32()
        self._check(self.lib.gpudb_q13_distribution(self.ctx, C.byref(cu.struct()), C.byref(od.struct()), C.byref(p),
                                                    rows, capacity, C.byref(n),
                                                    C.byref(timing) if timing is not None else None, None))
        return [(r.c_count, r.custdist) for r in rows[:min(n.value, capacity)]]

    def q9(self, pa, su, ps, od, li, smem_slots=0, global_slots=0, chunk_rows=0, capacity=4096, timing=None):
        """[(nation, year, profit)] ordered by nation asc, year desc."""
        p = capi.Q9Params(smem_slots, global_slots, chunk_rows)
        groups = (capi.Q9Group * capacity)()
        n = C.c_uint32()
        ls = li if isinstance(li, capi.Lineitem) else li.lineitem()
        self._check(self.lib.gpudb_q9_star(self.ctx, C.byref(pa.struct()), C.byref(su.struct()),
                                           C.byref(ps.struct()), C.byref(od.struct()), C.byref(ls), C.byref(p),
                                           groups, capacity, C.byref(n),
                                           C.byref(timing) if timing is not None else None, None))
        return [(g.nation, g.year, g.profit) for g in groups[:min(n.value, capacity)]], n.value

    def select_lt(self, col_ptr, n, value, bits_ptr=None, rows_ptr=None, timing=None):
        cnt = C.c_uint64()
        self._check(self.lib.gpudb_select_lt(self.ctx, col_ptr, n, value, bits_ptr, rows_ptr, C.byref(cnt),
                                             C.byref(timing) if timing is not None else None, None))
        return cnt.value

    def sum_i32(self, col_ptr, n, timing=None):
        s = C.c_int64()
        self._check(self.lib.gpudb_sum_i32(self.ctx, col_ptr, n, C.byref(s),
                                           C.byref(timing) if timing is not None else None, None))
        return s.value

    def hash_join_count(self, build_ptr, nb, probe_ptr, np_, mode=capi.JOIN_GLOBAL, timing=None):
        m = C.c_uint64()
        self._check(self.lib.gpudb_hash_join_count(self.ctx, build_ptr, nb, probe_ptr, np_, mode, C.byref(m),
                                                   C.byref(timing) if timing is not None else None, None))
        return m.value

    def radix_partition(self, keys_ptr, payload_ptr, n, bits, keys_out, payload_out, offsets, timing=None):
        self._check(self.lib.gpudb_radix_partition(self.ctx, keys_ptr, payload_ptr, n, bits, keys_out, payload_out,
                                                   offsets, C.byref(timing) if timing is not None else None, None))

    def radix_join_pairs(self, build_ptr, nb, probe_ptr, np_, out_b, out_p, capacity, timing=None):
        m = C.c_uint64()
        self._check(self.lib.gpudb_radix_join_pairs(self.ctx, build_ptr, nb, probe_ptr, np_, out_b, out_p, capacity,
                                                    C.byref(m), C.byref(timing) if timing is not None else None, None))
        return m.value

    # ---- raw device buffers ---------------------------------------------------------------
    def device_array(self, nbytes):
        return self._alloc(nbytes, MEM_DEVICE)

    def device_free(self, ptr):
        self.lib.gpudb_device_free(self.ctx, ptr)

    def to_device(self, arr):
        a = np.ascontiguousarray(arr)
        p = self._alloc(a.nbytes, MEM_DEVICE)
        if a.nbytes:
            self._check(self.lib.gpudb_copy(self.ctx, p, a.ctypes.data, a.nbytes))
        return p

    def to_host(self, ptr, n, dtype):
        out = np.empty(n, dtype=dtype)
        if out.nbytes:
            self._check(self.lib.gpudb_copy(self.ctx, out.ctypes.data, ptr, out.nbytes))
        return out


def q1_to_dict(r):
    out = {}
    for g in r.groups[:r.n_groups]:
        out[(g.flag, g.status)] = dict(count=g.count, sum_qty=g.sum_qty.value(), sum_base_price=g.sum_base_price.value(),
                                       sum_disc_price=g.sum_disc_price.value(), sum_charge=g.sum_charge.value(),
                                       sum_discount=g.sum_discount.value())
    return out


def q3_to_list(r):
    return [(x.order_key, x.order_date, x.revenue) for x in r.rows[:r.n_rows]], r.n_groups
