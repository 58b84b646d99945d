/*
 * gpudb_capi.h -- C ABI of the B200 columnar query engine.
 *
 * One call per operator pipeline of the reference benchmark (nd-tung/GPUDBMetalBenchmark),
 * which exposes each pipeline as `void runQnBenchmark(MTL::Device*, MTL::CommandQueue*,
 * MTL::Library*)` (declared at src/infra.h:874-922, registered by name at
 * src/main.cpp:158-188) and binds kernel arguments by `[[buffer(i)]]` index. Here the
 * driver-level surface is the same set of pipelines, but every argument is a plain pointer
 * or a plain-old-data struct, so any FFI (ctypes, cgo, JNI, N-API) can bind it.
 *
 * Conventions
 *  - Every function returns int: GPUDB_OK (0) or a negative GPUDB_E_* code. The message of
 *    the last failure on a context is returned by gpudb_last_error_string(). (The reference
 *    prints to stderr and returns void, e.g. src/infra.h:178-186.)
 *  - Column pointers are device pointers unless a struct's `location` says
 *    GPUDB_MEM_HOST. A fact table in host memory is streamed to the GPU in chunks
 *    (the reference's chunkedStreamLoop, src/infra.h:816-869).
 *  - All arithmetic is exact integer arithmetic: money is int64 hundredths, products are
 *    accumulated in int64 and group totals in int128.
 *  - A context is thread-compatible: one host thread at a time per context.
 *  - Calls are synchronous unless gpudb_exec.async is set; async calls complete, and fill
 *    their host result structs, at the next gpudb_sync() on the context.
 */
#ifndef GPUDB_CAPI_H
#define GPUDB_CAPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GPUDB_ABI_VERSION 1

/* ---- status codes ------------------------------------------------------------------- */
enum {
  GPUDB_OK = 0,
  GPUDB_E_INVALID = -1,     /* bad argument (null pointer, size, alignment, parameter) */
  GPUDB_E_CUDA = -2,        /* a CUDA runtime call failed */
  GPUDB_E_OOM = -3,         /* device or pinned-host allocation failed */
  GPUDB_E_NODEVICE = -4,    /* no CUDA device, or not an sm_100 device */
  GPUDB_E_CAPACITY = -5,    /* a hash table or partition overflowed on the device */
  GPUDB_E_KEY_RANGE = -6,   /* a key outside the declared key range was seen on the device */
  GPUDB_E_TIMEOUT = -7,     /* a bounded device-side wait ran out */
  GPUDB_E_BUSY = -8,        /* serving: the request does not fit the admission budget */
  GPUDB_E_CLOSED = -9,      /* serving: the request loop is closed */
  GPUDB_E_UNSUPPORTED = -10
};

enum { GPUDB_MEM_DEVICE = 0, GPUDB_MEM_HOST = 1 };
/* Join modes. GLOBAL: one open-addressing hash table; RADIX: both sides hash-partitioned,
 * each partition joined in shared memory; DIRECT (Q3): an order-key bitmap and a direct map
 * key -> slot, the reference's orders_map (kernels/q3.metal:59-78); AUTO (Q3): DIRECT when the
 * map of the orders' key range fits 30% of device memory (the reference's rule,
 * src/q3.cpp:246), else GLOBAL. */
enum { GPUDB_JOIN_GLOBAL = 0, GPUDB_JOIN_RADIX = 1, GPUDB_JOIN_DIRECT = 2, GPUDB_JOIN_AUTO = 3 };

typedef struct gpudb_ctx gpudb_ctx;

/* Signed 128-bit integer as two 64-bit halves (value = hi * 2^64 + lo). */
typedef struct gpudb_i128 { uint64_t lo; int64_t hi; } gpudb_i128;

/* Per-call execution options (NULL = synchronous on the context's stream). A context's
 * calls share its scratch memory, so async calls of one context on DIFFERENT streams must
 * not overlap on the device; use one context per concurrent stream (as the serving lanes
 * do). Calls on one stream are ordered by the stream. */
typedef struct gpudb_exec {
  int32_t async;      /* 1: enqueue only; results land at the next gpudb_sync() */
  int32_t flags;      /* reserved, 0 */
  void* stream;       /* cudaStream_t to launch on; NULL = the context's stream */
} gpudb_exec;

/* Timing of one call, filled when the call completes. gpu_ms is measured with CUDA events
 * on the launching stream around all of the call's device work (copies included). */
typedef struct gpudb_timing {
  double gpu_ms;
  double host_ms;          /* wall time of the call on the host */
  uint64_t h2d_bytes;
  uint64_t d2h_bytes;
  uint32_t kernels;        /* kernel launches issued by the call */
  uint32_t chunks;         /* streamed chunks (0 for HBM-resident inputs) */
} gpudb_timing;

/* ---- lifecycle (replaces the device/queue/library setup of src/main.cpp:76-156) -------- */
int gpudb_create(int device, gpudb_ctx** out);
int gpudb_destroy(gpudb_ctx* ctx);
const char* gpudb_last_error_string(const gpudb_ctx* ctx);
int gpudb_abi_version(void);
/* Waits for all work enqueued on the context and completes pending async results. */
int gpudb_sync(gpudb_ctx* ctx);
/* The context's CUDA stream (a cudaStream_t), for callers that time or order work. */
void* gpudb_stream(gpudb_ctx* ctx);
/* Number of kernels this context has launched since creation. */
uint64_t gpudb_kernel_launches(const gpudb_ctx* ctx);
/* Context options (replaces the fixed ChunkConfig sizing of src/infra.h:42-57). */
enum {
  GPUDB_OPT_CHUNK_ROWS = 1,  /* rows per streamed chunk of a host-resident fact table (default 64M) */
  GPUDB_OPT_SCAN_VARIANT = 2, /* Q1 scan kernel: 0 auto (7), 1 TMA 2048-row tiles x 4 stages, 2 128-bit loads,
                                 3 one row per thread, 4 TMA 4096-row tiles x 2 stages, 5 TMA ring,
                                 6 TMA ring + shared accumulators, 7 128-bit loads + shared accumulators,
                                 8 as 7 with registers for three blocks per SM, 9 as 7 with four
                                 quads per thread per step, 10 as 7 with one quad per step and
                                 four blocks per SM */
  GPUDB_OPT_Q6_VARIANT = 3,   /* Q6 scan kernel: 0 auto (1 below 2^24 rows, else 2), 1 one row per thread,
                                 2/3/4 128-bit loads with 1/2/4 quads (4/8/16 rows) per thread per step */
  GPUDB_OPT_HT_LOAD = 4,      /* largest load of the Q3/Q9 build hash tables, percent: 50 (default) or 25 */
  GPUDB_OPT_RADIX_BITS = 5,   /* Q3 radix mode fan-out (bits) when a call's radix_bits is 0; 0 = from the
                                 build size, ~4096 build rows per partition (default) */
  GPUDB_OPT_Q9_SMEM_SLOTS = 6,   /* Q9 per-block aggregation slots when a call's smem_slots is 0 (1024) */
  GPUDB_OPT_Q9_GLOBAL_SLOTS = 7, /* Q9 global aggregation slots when a call's global_slots is 0 (4096) */
  GPUDB_OPT_GRAPHS = 8           /* 1 (default): a Q9 call over device-resident tables on the context's
                                    stream is captured into a CUDA graph once per (tables, parameters)
                                    and replayed after; 0: its kernels are launched one by one */,
  GPUDB_OPT_RADIX_SHAPE = 10,    /* radix scatter block shape: 1 512 threads x 16 rows, 2 256 x 8 (both
                                    loading rows directly), 3 512 x 8, 4 256 x 8, 5 512 x 16, 7 256 x 16
                                    (each with a two-stage bulk-copy ring of sub-tiles), 6 512 x 16 with
                                    a one-stage ring; 0 (default) = 5. A shape whose shared memory does
                                    not fit falls back to 3, 4, then 2 */
  GPUDB_OPT_Q3_AUTO_MODE = 9     /* what a Q3 call with join_mode GPUDB_JOIN_AUTO runs: -1 (default) the
                                    30% rule (direct map when it fits, else the global table), or
                                    GPUDB_JOIN_GLOBAL / _RADIX / _DIRECT (the autotuner's choice) */
};
int gpudb_set_option(gpudb_ctx* ctx, int32_t option, int64_t value);
int gpudb_get_option(const gpudb_ctx* ctx, int32_t option, int64_t* value);

/* ---- memory (replaces MTL::Device::newBuffer and createFilledBuffer, src/infra.h:527-531) */
int gpudb_device_alloc(gpudb_ctx* ctx, size_t bytes, void** out);
int gpudb_device_free(gpudb_ctx* ctx, void* p);
int gpudb_host_alloc(gpudb_ctx* ctx, size_t bytes, void** out);     /* pinned host memory */
int gpudb_host_free(gpudb_ctx* ctx, void* p);
int gpudb_copy(gpudb_ctx* ctx, void* dst, const void* src, size_t bytes); /* any direction */

/* ---- column sets ------------------------------------------------------------------------ */
/* Fact table (the reference's lineitem columns). Unused columns may be NULL. key_max fields
 * give the largest key value of a join key column, used to size bitmaps and direct maps. */
typedef struct gpudb_lineitem {
  uint64_t n_rows;
  int32_t location;            /* GPUDB_MEM_DEVICE or GPUDB_MEM_HOST */
  int32_t order_key_max;
  const int32_t* ship_date;    /* day number, 0 = first day of the date domain */
  const int32_t* quantity;
  const int64_t* ext_price;    /* hundredths */
  const int32_t* discount;     /* hundredths: 0..10 means 0.00..0.10 */
  const int32_t* tax;          /* hundredths */
  const uint8_t* flag;         /* 0..2 */
  const uint8_t* status;       /* 0..1 */
  const int32_t* order_key;
  const int32_t* part_key;
  const int32_t* supp_key;
  const int32_t* commit_date;  /* day number (Q4, Q12) */
  const int32_t* receipt_date; /* day number (Q4, Q12) */
  const uint8_t* ship_mode;    /* GPUDB_MODE_*: 0..6 (Q12) */
} gpudb_lineitem;

/* l_shipmode codes, in the order of the strings (ORDER BY l_shipmode) */
enum { GPUDB_MODE_AIR = 0, GPUDB_MODE_FOB, GPUDB_MODE_MAIL, GPUDB_MODE_RAIL, GPUDB_MODE_REG_AIR,
       GPUDB_MODE_SHIP, GPUDB_MODE_TRUCK };

typedef struct gpudb_customer {
  uint64_t n_rows; int32_t key_max; int32_t reserved;
  const int32_t* cust_key; const uint8_t* segment;
  const uint8_t* nation;       /* c_nationkey 0..24 (Q5) */
} gpudb_customer;

typedef struct gpudb_orders {
  uint64_t n_rows; int32_t key_max; int32_t cust_key_max;
  const int32_t* order_key; const int32_t* cust_key; const int32_t* order_date;
  const uint8_t* priority;     /* o_orderpriority 1..5 = '1-URGENT' .. '5-LOW' (Q4, Q12) */
  const char* comment;         /* o_comment: GPUDB_COMMENT_WIDTH bytes per row, NUL-padded (Q13) */
} gpudb_orders;
#define GPUDB_COMMENT_WIDTH 80   /* at most 79 characters; the bytes after the text are 0 */

typedef struct gpudb_part {
  uint64_t n_rows; int32_t key_max; int32_t reserved;
  const int32_t* part_key; const uint8_t* flag;      /* flag != 0: the part passes the filter */
  const uint8_t* type;         /* p_type code 0..149 (Q8): see GPUDB_PART_TYPE */
} gpudb_part;
/* p_type code of "S1 S2 S3": s1 in STANDARD, SMALL, MEDIUM, LARGE, ECONOMY, PROMO; s2 in
 * ANODIZED, BURNISHED, PLATED, POLISHED, BRUSHED; s3 in TIN, NICKEL, BRASS, STEEL, COPPER
 * (0-based positions in those lists); "ECONOMY ANODIZED STEEL" = 103. */
#define GPUDB_PART_TYPE(s1, s2, s3) ((s1) * 25 + (s2) * 5 + (s3))

typedef struct gpudb_supplier {
  uint64_t n_rows; int32_t key_max; int32_t reserved;
  const int32_t* supp_key; const uint8_t* nation;
} gpudb_supplier;

typedef struct gpudb_partsupp {
  uint64_t n_rows;
  const int32_t* part_key; const int32_t* supp_key; const int64_t* supply_cost;
} gpudb_partsupp;

/* ---- synthetic data (replaces the .tbl loaders, src/infra.h:262-409) -------------------- */
enum gpudb_column_id {
  GPUDB_COL_LI_SHIP_DATE = 1, GPUDB_COL_LI_QUANTITY, GPUDB_COL_LI_EXT_PRICE,
  GPUDB_COL_LI_DISCOUNT, GPUDB_COL_LI_TAX, GPUDB_COL_LI_FLAG, GPUDB_COL_LI_STATUS,
  GPUDB_COL_LI_ORDER_KEY, GPUDB_COL_LI_PART_KEY, GPUDB_COL_LI_SUPP_KEY,
  GPUDB_COL_LI_COMMIT_DATE, GPUDB_COL_LI_RECEIPT_DATE, GPUDB_COL_LI_SHIP_MODE,
  GPUDB_COL_CU_CUST_KEY = 20, GPUDB_COL_CU_SEGMENT, GPUDB_COL_CU_NATION,
  GPUDB_COL_OR_ORDER_KEY = 30, GPUDB_COL_OR_CUST_KEY, GPUDB_COL_OR_ORDER_DATE, GPUDB_COL_OR_PRIORITY,
  GPUDB_COL_OR_COMMENT,        /* GPUDB_COMMENT_WIDTH bytes per row */
  GPUDB_COL_PA_PART_KEY = 40, GPUDB_COL_PA_FLAG, GPUDB_COL_PA_TYPE,
  GPUDB_COL_SU_SUPP_KEY = 50, GPUDB_COL_SU_NATION,
  GPUDB_COL_PS_PART_KEY = 60, GPUDB_COL_PS_SUPP_KEY, GPUDB_COL_PS_SUPPLY_COST
};
enum { GPUDB_ORDERS_NONE = 0, GPUDB_ORDERS_CLUSTERED = 1, GPUDB_ORDERS_UNIFORM = 2 };

typedef struct gpudb_gen_spec {
  uint64_t seed;
  uint64_t row_offset;         /* first row to generate (chunks and shards) */
  uint64_t n_rows;             /* rows to generate */
  int64_t n_orders;            /* orders table size (lineitem order keys) */
  int64_t n_cust;              /* customer table size (orders cust keys) */
  int64_t n_parts;             /* part table size */
  int64_t n_supp;              /* supplier table size (a multiple of 4) */
  int32_t order_mode;          /* GPUDB_ORDERS_* for lineitem order keys */
  int32_t reserved;
} gpudb_gen_spec;

/* Writes rows [row_offset, row_offset+n_rows) of one column to dst, which is device memory
 * (location GPUDB_MEM_DEVICE, generated by a kernel) or host memory (GPUDB_MEM_HOST,
 * generated on the host cores). Both produce identical bytes. */
int gpudb_generate(gpudb_ctx* ctx, const gpudb_gen_spec* spec, int32_t column,
                   void* dst, int32_t location);
/* Element size in bytes of a generated column, or 0 for an unknown column. */
int gpudb_column_width(int32_t column);

/* ---- Q6-like filtered sum (replaces runQ6Benchmark src/q6.cpp:8-120 and kernels
 *      q6_filter_and_sum_stage1/2 kernels/q6.metal:12-70; streamed form replaces
 *      runQ6BenchmarkSF100 src/q6.cpp:124-214) --------------------------------------- */
typedef struct gpudb_q6_params {
  int32_t ship_lo, ship_hi;    /* ship_date in [ship_lo, ship_hi) */
  int32_t disc_lo, disc_hi;    /* discount in [disc_lo, disc_hi] */
  int32_t qty_lt;              /* quantity < qty_lt */
} gpudb_q6_params;
typedef struct gpudb_q6_result { int64_t revenue; uint64_t rows_matched; } gpudb_q6_result;
/* revenue = sum(ext_price * discount) over matching rows, in hundredths^2. */
int gpudb_q6_sum(gpudb_ctx* ctx, const gpudb_lineitem* li, const gpudb_q6_params* p,
                 gpudb_q6_result* out, gpudb_timing* t, const gpudb_exec* ex);

/* Q6-like filtered sum that allocates nothing. No counterpart in the reference: it exists
 * for callers that cannot call cudaMalloc -- programs whose device memory is owned and
 * budgeted by another memory manager (a server that hands out all of the GPU), and plugins
 * that have no gpudb_ctx (the context owns every other call's scratch memory). It needs no
 * context. li must be device-resident; `out` is a
 * caller-owned device buffer of two int64 (revenue, rows matched) that the call overwrites;
 * the work is enqueued on `stream` (a cudaStream_t, NULL = default stream) of the current
 * device and the call does not wait for it. Scratch is a fixed 262,400-byte static device
 * array that every GPU loading this library holds until exit, so li->n_rows is limited to
 * 67,108,864 rows (GPUDB_E_CAPACITY beyond). The first call on a device looks up that
 * array's device address (cudaGetSymbolAddress); make that first call before any stream
 * capture. The address is kept for the life of the process, so a device reset after that
 * first call is not supported. All calls on a device share the one array: calls that
 * overlap on the GPU (for example on two streams at once) race and give wrong results. A
 * launch failure returns GPUDB_E_CUDA; an error already pending from the caller's own
 * earlier CUDA work is left in place for the caller. */
int gpudb_q6_sum_noalloc(const gpudb_lineitem* li, const gpudb_q6_params* p, int64_t* out, void* stream);

/* ---- Q1-like filter + 6-group aggregate (replaces runQ1Benchmark src/q1.cpp:8-173 and
 *      q1_fused_kernel kernels/q1.metal:39-121; streamed form replaces runQ1BenchmarkSF100
 *      src/q1.cpp:177-376) ------------------------------------------------------------ */
typedef struct gpudb_q1_params { int32_t ship_le; int32_t reserved; } gpudb_q1_params;
typedef struct gpudb_q1_group {
  uint8_t flag, status; uint8_t reserved[6];
  uint64_t count;
  gpudb_i128 sum_qty;
  gpudb_i128 sum_base_price;   /* sum(ext_price), hundredths */
  gpudb_i128 sum_disc_price;   /* sum(ext_price*(100-discount)), hundredths^2 */
  gpudb_i128 sum_charge;       /* sum(ext_price*(100-discount)*(100+tax)), hundredths^3 */
  gpudb_i128 sum_discount;     /* sum(discount), hundredths (for avg_disc) */
} gpudb_q1_group;
typedef struct gpudb_q1_result {
  uint32_t n_groups; uint32_t reserved;
  gpudb_q1_group groups[6];    /* non-empty groups in (flag, status) order */
} gpudb_q1_result;
int gpudb_q1_group6(gpudb_ctx* ctx, const gpudb_lineitem* li, const gpudb_q1_params* p,
                    gpudb_q1_result* out, gpudb_timing* t, const gpudb_exec* ex);

/* ---- Q3-like bitmap semi-join + hash join + per-order aggregate + top-k (replaces
 *      runQ3Benchmark src/q3.cpp:8-173, kernels q3_build_customer_bitmap_kernel,
 *      q3_build_orders_map_kernel/_ht_kernel, q3_probe_and_aggregate_*_kernel,
 *      q3_compact_results_kernel kernels/q3.metal:43-340, and sortAndPrintQ3
 *      src/infra.h:538-564; streamed form replaces runQ3BenchmarkSF100 src/q3.cpp:177-538) */
#define GPUDB_Q3_MAX_K 64
typedef struct gpudb_q3_params {
  int32_t segment;             /* customer.segment == segment */
  int32_t order_date_lt;       /* orders.order_date < order_date_lt */
  int32_t ship_date_gt;        /* lineitem.ship_date > ship_date_gt */
  int32_t k;                   /* rows of the top-k, 1..GPUDB_Q3_MAX_K */
  int32_t join_mode;           /* GPUDB_JOIN_GLOBAL, _RADIX, _DIRECT (needs orders.key_max) or _AUTO */
  int32_t radix_bits;          /* radix mode: partition bits, 0 = chosen from the build size */
} gpudb_q3_params;
typedef struct gpudb_q3_row { int32_t order_key; int32_t order_date; int64_t revenue; } gpudb_q3_row;
/* Rows ordered by revenue desc, order_date asc, order_key asc. revenue is in hundredths^2. */
typedef struct gpudb_q3_result {
  uint64_t n_groups;           /* orders with at least one joined lineitem row */
  uint32_t n_rows;
  int32_t join_mode;           /* the mode that ran (AUTO resolved) */
  gpudb_q3_row rows[GPUDB_Q3_MAX_K];
} gpudb_q3_result;
int gpudb_q3_join_topk(gpudb_ctx* ctx, const gpudb_customer* cu, const gpudb_orders* od,
                       const gpudb_lineitem* li, const gpudb_q3_params* p,
                       gpudb_q3_result* out, gpudb_timing* t, const gpudb_exec* ex);

/* ---- Q9-like star join + (nation, year) aggregate (replaces runQ9Benchmark
 *      src/q9.cpp:8-241, kernels q9_build_*_kernel and q9_probe_and_global_agg_kernel
 *      kernels/q9.metal:44-289, postProcessQ9 src/infra.h:743-776; streamed form replaces
 *      runQ9BenchmarkSF100 src/q9.cpp:245-557 and q9_probe_directorders_kernel
 *      kernels/q9.metal:308-394) ------------------------------------------------------ */
typedef struct gpudb_q9_params {
  int32_t smem_slots;          /* per-block aggregation slots, 0 = default (power of two) */
  int32_t global_slots;        /* global aggregation table slots, 0 = default (power of two) */
  uint64_t chunk_rows;         /* host-resident lineitem: rows per streamed chunk, 0 = default;
                                  also the rows per filter + resolve piece (at most 64M) */
} gpudb_q9_params;
typedef struct gpudb_q9_group { int32_t nation; int32_t year; int64_t profit; } gpudb_q9_group;
/* profit = sum(ext_price*(100-discount) - supply_cost*quantity*100), hundredths^2.
 * Groups are ordered by nation asc, year desc; *n_groups is the total number of groups and
 * at most `capacity` of them are written. */
int gpudb_q9_star(gpudb_ctx* ctx, const gpudb_part* pa, const gpudb_supplier* su,
                  const gpudb_partsupp* ps, const gpudb_orders* od, const gpudb_lineitem* li,
                  const gpudb_q9_params* p, gpudb_q9_group* out, uint32_t capacity,
                  uint32_t* n_groups, gpudb_timing* t, const gpudb_exec* ex);

/* ---- Q4 order priority checking (replaces runQ4Benchmark src/q4.cpp:8-127 and its kernels
 *      q4_build_late_bitmap / q4_count_by_priority_stage1 / q4_final_count_stage2
 *      kernels/q4.metal:21-94; the streamed form replaces runQ4BenchmarkSF100
 *      src/q4.cpp:130-282) ------------------------------------------------------------------
 * count[p - 1] = number of orders with priority p (1..5) and date_lo <= order_date < date_hi
 * that have a lineitem row with commit_date < receipt_date (EXISTS). The "late" bitmap covers
 * order keys 0..od->key_max; lineitem keys outside it match no order. Lineitem may be
 * host-resident (streamed in chunks). */
typedef struct gpudb_q4_params { int32_t date_lo; int32_t date_hi; } gpudb_q4_params;
typedef struct gpudb_q4_result { uint64_t count[5]; } gpudb_q4_result;
int gpudb_q4_priority(gpudb_ctx* ctx, const gpudb_orders* od, const gpudb_lineitem* li, const gpudb_q4_params* p,
                      gpudb_q4_result* out, gpudb_timing* t, const gpudb_exec* ex);

/* ---- Q12 shipping modes and order priority (replaces runQ12Benchmark src/q12.cpp:8-125 and
 *      its kernels q12_build_priority_bitmap / q12_filter_and_count_stage1 /
 *      q12_final_count_stage2 kernels/q12.metal:22-99; the streamed form replaces
 *      runQ12BenchmarkSF100 src/q12.cpp:128-277) --------------------------------------------
 * For lineitem rows with ship_mode == mode[m] (m = 0, 1), receipt_lo <= receipt_date <
 * receipt_hi, commit_date < receipt_date and ship_date < commit_date: high[m] counts the rows
 * whose order has priority 1..high_max (the query's '1-URGENT', '2-HIGH': high_max = 2), low[m]
 * the others (as the reference's priority bitmap does: a row whose order key is outside
 * 0..od->key_max or has no order counts as low). */
typedef struct gpudb_q12_params {
  int32_t receipt_lo; int32_t receipt_hi; int32_t mode[2]; int32_t high_max; int32_t reserved;
} gpudb_q12_params;
typedef struct gpudb_q12_result { uint64_t high[2]; uint64_t low[2]; } gpudb_q12_result;
int gpudb_q12_shipmode(gpudb_ctx* ctx, const gpudb_orders* od, const gpudb_lineitem* li, const gpudb_q12_params* p,
                       gpudb_q12_result* out, gpudb_timing* t, const gpudb_exec* ex);

/* ---- Q5 local supplier volume (replaces runQ5Benchmark src/q5.cpp:8-200 with its kernels
 *      q5_build_customer_nation_map_kernel / q5_build_supplier_nation_map_kernel /
 *      q5_build_orders_map_kernel / q5_probe_and_aggregate_kernel kernels/q5.metal:19-125) -------
 * revenue[n] = sum of ext_price * (100 - discount) (hundredths^2) over lineitem rows whose order
 * has date_lo <= order_date < date_hi, whose customer and supplier are both of nation n, and n
 * is in nation_mask (bit n: the nations of the region, e.g. ASIA = 8, 9, 12, 18, 21). Customer,
 * supplier and order keys outside their tables' 0..key_max fail with GPUDB_E_KEY_RANGE;
 * lineitem keys outside them match nothing. Lineitem may be host-resident (streamed). */
#define GPUDB_NATIONS 25
typedef struct gpudb_q5_params { int32_t date_lo; int32_t date_hi; uint32_t nation_mask; int32_t reserved; } gpudb_q5_params;
typedef struct gpudb_q5_result { int64_t revenue[GPUDB_NATIONS]; } gpudb_q5_result;
int gpudb_q5_local_supplier(gpudb_ctx* ctx, const gpudb_customer* cu, const gpudb_supplier* su, const gpudb_orders* od,
                            const gpudb_lineitem* li, const gpudb_q5_params* p, gpudb_q5_result* out,
                            gpudb_timing* t, const gpudb_exec* ex);

/* ---- Q7 volume shipping (replaces runQ7Benchmark src/q7.cpp with its kernels
 *      q7_build_supplier_map_kernel / q7_build_customer_map_kernel / q7_build_orders_map_kernel /
 *      q7_probe_and_aggregate_kernel kernels/q7.metal:12-109) ----------------------------------
 * For lineitem rows with ship_lo <= ship_date <= ship_hi (both ends included, at most
 * GPUDB_MAX_YEARS calendar years) whose supplier and whose order's customer are of nations
 * (a, b) or (b, a): revenue[pair][y] += ext_price * (100 - discount), pair 0 = supplier of a
 * and customer of b, pair 1 = supplier of b and customer of a, y = calendar year of the ship
 * date - first_year. Keys outside their tables' 0..key_max fail with GPUDB_E_KEY_RANGE (lineitem
 * keys outside them match nothing). Lineitem may be host-resident (streamed). */
#define GPUDB_MAX_YEARS 8
typedef struct gpudb_q7_params { int32_t nation_a; int32_t nation_b; int32_t ship_lo; int32_t ship_hi; } gpudb_q7_params;
typedef struct gpudb_q7_result {
  int32_t first_year; int32_t n_years; int64_t revenue[2][GPUDB_MAX_YEARS];
} gpudb_q7_result;
int gpudb_q7_volume_shipping(gpudb_ctx* ctx, const gpudb_customer* cu, const gpudb_supplier* su, const gpudb_orders* od,
                             const gpudb_lineitem* li, const gpudb_q7_params* p, gpudb_q7_result* out,
                             gpudb_timing* t, const gpudb_exec* ex);

/* ---- Q8 national market share (replaces runQ8Benchmark src/q8.cpp with its kernels
 *      q8_build_orders_map_kernel / q8_probe_and_aggregate_kernel kernels/q8.metal:9-76) -------
 * For lineitem rows whose part has type part_type and whose order has date_lo <= order_date <=
 * date_hi (both included, at most GPUDB_MAX_YEARS calendar years) and a customer of a nation in
 * region_mask: volume[y] += ext_price * (100 - discount), and nation_volume[y] too when the
 * supplier is of `nation`; y = calendar year of the order date - first_year. The market share
 * of year y is nation_volume[y] / volume[y]. Key errors as for Q7. */
typedef struct gpudb_q8_params {
  int32_t date_lo; int32_t date_hi; uint32_t region_mask; int32_t nation; int32_t part_type; int32_t reserved;
} gpudb_q8_params;
typedef struct gpudb_q8_result {
  int32_t first_year; int32_t n_years; int64_t volume[GPUDB_MAX_YEARS]; int64_t nation_volume[GPUDB_MAX_YEARS];
} gpudb_q8_result;
int gpudb_q8_market_share(gpudb_ctx* ctx, const gpudb_customer* cu, const gpudb_supplier* su, const gpudb_part* pa,
                          const gpudb_orders* od, const gpudb_lineitem* li, const gpudb_q8_params* p,
                          gpudb_q8_result* out, gpudb_timing* t, const gpudb_exec* ex);

/* ---- Q10 returned item reporting (replaces runQ10Benchmark src/q10.cpp:8-140 with its kernels
 *      q10_build_orders_map_kernel / q10_probe_and_aggregate_kernel kernels/q10.metal:8-54 and
 *      its host top-20 heap src/q10.cpp:102-121) ------------------------------------------------
 * revenue(customer) = sum of ext_price * (100 - discount) (hundredths^2) over lineitem rows with
 * flag 2 ('R', returned) whose order has date_lo <= order_date < date_hi and belongs to a
 * customer of `cu`. rows[] = the k (1..GPUDB_Q3_MAX_K) customers of largest revenue, ordered
 * by revenue desc then cust_key asc; n_customers = customers with revenue > 0. An order key
 * outside 0..od->key_max or a customer key outside 0..cu->key_max in the tables fails with
 * GPUDB_E_KEY_RANGE; an order of a customer that is not in `cu` and a lineitem row of an
 * order outside the window count for nobody. Lineitem may be host-resident (streamed). */
typedef struct gpudb_q10_params { int32_t date_lo; int32_t date_hi; int32_t k; int32_t reserved; } gpudb_q10_params;
typedef struct gpudb_q10_row { int32_t cust_key; int32_t reserved; int64_t revenue; } gpudb_q10_row;
typedef struct gpudb_q10_result {
  uint64_t n_customers;
  uint32_t n_rows;
  uint32_t reserved;
  gpudb_q10_row rows[GPUDB_Q3_MAX_K];
} gpudb_q10_result;
int gpudb_q10_returned(gpudb_ctx* ctx, const gpudb_customer* cu, const gpudb_orders* od, const gpudb_lineitem* li,
                       const gpudb_q10_params* p, gpudb_q10_result* out, gpudb_timing* t, const gpudb_exec* ex);

/* ---- Q13 customer distribution (replaces runQ13Benchmark src/q13.cpp:8-117 with its kernels
 *      q13_pattern_match_kernel / q13_count_prefiltered_kernel / q13_build_histogram_kernel
 *      kernels/q13.metal:33-168 and postProcessQ13 src/infra.h:778-800) -------------------------
 * c_count(customer) = number of its orders whose comment is NOT LIKE '%word1%word2%' (word1
 * followed, later in the comment, by word2; 1..15 characters each, NUL-terminated); custdist =
 * number of customers per c_count, over every row of `cu` (customers without such orders have
 * c_count 0: the LEFT OUTER JOIN). Rows are ordered by custdist desc, c_count desc; *n_rows is
 * the number of distinct c_count values and at most `capacity` rows are written. Orders whose
 * customer key is outside 0..cu->key_max count for no customer; a c_count above
 * GPUDB_Q13_MAX_COUNT fails the call with GPUDB_E_CAPACITY. */
#define GPUDB_Q13_MAX_COUNT 1023
typedef struct gpudb_q13_params { char word1[16]; char word2[16]; } gpudb_q13_params;
typedef struct gpudb_q13_row { uint32_t c_count; uint32_t custdist; } gpudb_q13_row;
int gpudb_q13_distribution(gpudb_ctx* ctx, const gpudb_customer* cu, const gpudb_orders* od,
                           const gpudb_q13_params* p, gpudb_q13_row* out, uint32_t capacity, uint32_t* n_rows,
                           gpudb_timing* t, const gpudb_exec* ex);

/* ---- microbenchmarks (replace runSelectionBenchmark / runAggregationBenchmark /
 *      runJoinBenchmark src/microbenchmarks.cpp:8-251 and their kernels
 *      kernels/microbenchmarks.metal:160-294) ------------------------------------------ */
/* Rows with col[i] < value. out_bits (nullable, (n+31)/32 device words) receives a row
 * bitmask; out_rows (nullable, device, capacity n) receives matching row ids in order. */
int gpudb_select_lt(gpudb_ctx* ctx, const int32_t* col, uint64_t n, int32_t value,
                    uint32_t* out_bits, uint32_t* out_rows, uint64_t* count,
                    gpudb_timing* t, const gpudb_exec* ex);
/* Exact int64 sum of an int32 column. */
int gpudb_sum_i32(gpudb_ctx* ctx, const int32_t* col, uint64_t n, int64_t* sum,
                  gpudb_timing* t, const gpudb_exec* ex);
/* Number of probe rows whose key occurs among the build keys (hash_join_probe counts a
 * probe row once, at its first match). mode: GPUDB_JOIN_GLOBAL (one hash set), GPUDB_JOIN_RADIX
 * (radix partitions, a shared-memory set per partition) or GPUDB_JOIN_DIRECT (one bit per key
 * of the build keys' span [min, max], found on the device; a span of 2^30 keys or more
 * returns GPUDB_E_KEY_RANGE; the context keeps 128 MB of scratch for the bits). */
int gpudb_hash_join_count(gpudb_ctx* ctx, const int32_t* build_keys, uint64_t n_build,
                          const int32_t* probe_keys, uint64_t n_probe, int32_t mode,
                          uint64_t* matches, gpudb_timing* t, const gpudb_exec* ex);

/* ---- radix partitioning (replaces sf100_radix_histogram / _prefix_sum / _scatter /
 *      sf100_partition_join kernels/microbenchmarks.metal:15-156) ---------------------- */
/* Partition p of a key is hash(key) & (2^bits - 1) with the reference's key hash
 * (sf100_hash_key, kernels/common.h:81-87). Rows keep their input order inside a
 * partition. offsets receives 2^bits + 1 device words (exclusive prefix of the sizes). */
int gpudb_radix_partition(gpudb_ctx* ctx, const int32_t* keys, const int32_t* payload,
                          uint64_t n, int32_t bits, int32_t* keys_out, int32_t* payload_out,
                          uint32_t* offsets, gpudb_timing* t, const gpudb_exec* ex);
/* All (build row, probe row) pairs with equal keys, via radix partitioning and per-partition
 * shared-memory hash tables. Pairs are written in (probe row, build row) order; *n_pairs is
 * the total, at most `capacity` pairs are written (device arrays). */
int gpudb_radix_join_pairs(gpudb_ctx* ctx, const int32_t* build_keys, uint64_t n_build,
                           const int32_t* probe_keys, uint64_t n_probe,
                           int32_t* out_build_rows, int32_t* out_probe_rows,
                           uint64_t capacity, uint64_t* n_pairs,
                           gpudb_timing* t, const gpudb_exec* ex);

/* ---- batched execution (no reference counterpart: the reference runs one query per
 *      command buffer, src/q1.cpp:59-106) ---------------------------------------------
 * One call runs many requests, each with its own exact result and status:
 *  - Q6/Q1 requests over device-resident tables are grouped by (table, row range): one Q1
 *    request with up to 4 Q6 requests runs as one Q1 scan that evaluates the Q6 requests on
 *    the rows it reads; one or two Q1 (up to three Q6) requests alone run their own scans;
 *    more share passes that read the rows once (up to 8 Q6 per pass; up to 2 Q1 per pass,
 *    with 4 Q6 riding along), persistent launches that pull row tiles from a device queue;
 *  - Q6/Q1 requests over the same host-resident table share one chunked copy of it;
 *  - Q3 requests (global mode) over the same tables run in groups of up to 8 that share
 *    every stage's launch and one probe pass over the fact table;
 *  - in a synchronous call, identical Q3/Q9 requests run once and the others get copies;
 *  - a lone request runs through its own pipeline, exactly as the single-request call.
 * Everything is enqueued on one stream, cheapest work per request first (scans of tables of
 * at most 2^24 rows, the joins that run alone, the Q3 groups, scans of larger tables, scans
 * of host-resident tables), and each request completes when its own work has finished; a
 * synchronous call times the whole batch in `t`. */
enum { GPUDB_PIPE_Q6 = 1, GPUDB_PIPE_Q1 = 2, GPUDB_PIPE_Q3 = 3, GPUDB_PIPE_Q9 = 4 };

typedef struct gpudb_q3_tables { gpudb_customer cu; gpudb_orders od; gpudb_lineitem li; } gpudb_q3_tables;
typedef struct gpudb_q9_tables {
  gpudb_part pa; gpudb_supplier su; gpudb_partsupp ps; gpudb_orders od; gpudb_lineitem li;
} gpudb_q9_tables;

typedef struct gpudb_request {
  int32_t pipeline;                 /* GPUDB_PIPE_* */
  int32_t status;                   /* set when the request completes: GPUDB_OK or GPUDB_E_* */
  uint64_t row_begin, row_end;      /* Q6/Q1: rows [row_begin, row_end) of li; row_end 0 = all rows */
  const gpudb_lineitem* li;         /* Q6/Q1 input */
  const gpudb_q3_tables* q3;        /* Q3 input */
  const gpudb_q9_tables* q9;        /* Q9 input */
  gpudb_q6_params q6;
  gpudb_q1_params q1;
  gpudb_q3_params q3p;
  gpudb_q9_params q9p;
  gpudb_q6_result* q6_out;          /* caller-owned results, filled at completion */
  gpudb_q1_result* q1_out;
  gpudb_q3_result* q3_out;
  gpudb_q9_group* q9_out; uint32_t q9_capacity; uint32_t q9_groups;
} gpudb_request;

/* Runs n requests; with ex->async the requests complete (status and results filled) at the
 * next gpudb_sync(). Returns GPUDB_OK when the batch was accepted; per-request failures
 * are reported in each request's status. */
int gpudb_batch_run(gpudb_ctx* ctx, gpudb_request* reqs, uint32_t n, gpudb_timing* t, const gpudb_exec* ex);

/* ---- .tbl text loader (replaces MappedFile/countLines/buildLineIndex/parse*ColumnChunk,
 *      src/infra.h:60-171, and loadColumnsMulti, src/infra.h:262-361) ----------------------
 * Parses dbgen-style text ('|'-separated fields, one row per line, '\r' before the newline
 * allowed) on the GPU into the engine's columns. Encodings: integers as int32; decimals (at
 * most two fraction digits) as hundredths; dates "YYYY-MM-DD" as days since 1992-01-01;
 * return flag A/N/R -> 0/1/2; line status F/O -> 0/1; market segment AUTOMOBILE, BUILDING,
 * FURNITURE, HOUSEHOLD, MACHINERY -> 0..4; part name -> 1 if it contains "green"; ship mode
 * AIR, FOB, MAIL, RAIL, REG AIR, SHIP, TRUCK -> 0..6; order priority "1-URGENT".."5-LOW" -> 1..5. (The
 * reference keeps dates as YYYYMMDD ints and money as float.) Columns kept, in cols[] order,
 * with the dbgen fields they come from:
 *   LINEITEM: order_key, part_key, supp_key, quantity, ext_price (int64), discount, tax,
 *             flag (u8), status (u8), ship_date, commit_date, receipt_date, ship_mode (u8)
 *                                                     fields 0,1,2,4,5,6,7,8,9,10,11,12,14
 *   ORDERS:   order_key, cust_key, order_date, priority (u8), comment (GPUDB_COMMENT_WIDTH
 *             bytes per row: at most 79 characters, NUL-padded)    fields 0,1,4,5,8
 *   CUSTOMER: cust_key, nation (u8), segment (u8)                  fields 0,3,6
 *   PART:     part_key, flag (u8), type (u8, GPUDB_PART_TYPE)      fields 0,1,4
 *   SUPPLIER: supp_key, nation (u8)                                fields 0,3
 *   PARTSUPP: part_key, supp_key, supply_cost (int64)              fields 0,1,3
 * `cols` are device columns holding `capacity` rows (a NULL column is parsed and checked but
 * not stored). text is host memory (copied inside the call) or 16-byte aligned device memory.
 * Outputs: *n_rows, and col_max[i] (GPUDB_TBL_MAX_COLS entries, may be NULL) = the largest
 * value of int32 column i (INT32_MIN for other columns): the key bounds the join pipelines
 * take. A malformed field fails the call with GPUDB_E_INVALID; more rows than capacity with
 * GPUDB_E_CAPACITY. gpudb_tbl_count_rows counts the rows without parsing them. */
enum { GPUDB_TBL_LINEITEM = 1, GPUDB_TBL_ORDERS = 2, GPUDB_TBL_CUSTOMER = 3, GPUDB_TBL_PART = 4,
       GPUDB_TBL_SUPPLIER = 5, GPUDB_TBL_PARTSUPP = 6 };
#define GPUDB_TBL_MAX_COLS 13
int gpudb_tbl_count_rows(gpudb_ctx* ctx, const char* text, uint64_t bytes, int32_t location, uint64_t* n_rows);
int gpudb_tbl_parse(gpudb_ctx* ctx, int32_t table, const char* text, uint64_t bytes, int32_t location,
                    void* const* cols, uint64_t capacity, uint64_t* n_rows, int32_t* col_max,
                    gpudb_timing* t);

/* ---- self-test of the bounded device waits (no reference counterpart) ---------------------
 * One warp waits on a shared-memory mbarrier through the same bounded wait the TMA scan
 * kernels use. arrive != 0: a thread arrives first, the call returns GPUDB_OK. arrive == 0:
 * nothing arrives, the wait gives up after `polls` polls (1..2^26; it also stops after 2 s)
 * and the call returns GPUDB_E_TIMEOUT with the context still usable. */
int gpudb_selftest_bounded_wait(gpudb_ctx* ctx, uint32_t polls, int32_t arrive);

/* ---- autotuner (no reference counterpart) --------------------------------------------
 * gpudb_autotune times the candidate settings of one request's pipeline on the request's
 * own tables (one synchronous run, then reps runs issued back to back on the context's
 * stream: median device time) and sets the fastest on the context:
 *   Q1: GPUDB_OPT_SCAN_VARIANT 1..10 (block size, rows per thread, 128-bit loads, TMA
 *       staging, shared-memory accumulators); Q6: GPUDB_OPT_Q6_VARIANT 1..4 (row kernel or
 *       128-bit loads with 1/2/4 quads per thread per step); Q3 global mode:
 *       GPUDB_OPT_HT_LOAD 50/25; Q3 radix mode: GPUDB_OPT_RADIX_BITS; Q3 AUTO mode:
 *       GPUDB_OPT_Q3_AUTO_MODE (direct map, global table or radix partitions); Q9:
 *       GPUDB_OPT_Q9_SMEM_SLOTS x GPUDB_OPT_Q9_GLOBAL_SLOTS.
 * A candidate whose result differs from the default setting's is dropped. The choices of a
 * context are written by gpudb_tune_save as lines "device|pipeline|rows_log2|option|value"
 * (other devices' lines are kept) and applied by gpudb_tune_load (this device's lines). */
typedef struct gpudb_tune_result {
  int32_t pipeline;          /* GPUDB_PIPE_* tuned */
  uint32_t candidates;       /* settings timed, the default included */
  uint32_t dropped;          /* candidates rejected: unsupported, failing or a different result */
  int32_t option;            /* the chosen setting, now set on the context */
  int64_t value;
  int32_t option2;           /* a second option of the same choice (0 = none) */
  int32_t reserved;
  int64_t value2;
  double best_ms;            /* median device time with the chosen setting */
  double default_ms;         /* median device time with the default setting */
} gpudb_tune_result;
int gpudb_autotune(gpudb_ctx* ctx, const gpudb_request* req, uint32_t reps, gpudb_tune_result* out);
int gpudb_tune_save(gpudb_ctx* ctx, const char* path);
int gpudb_tune_load(gpudb_ctx* ctx, const char* path, uint32_t* applied);

/* ---- serving (no reference counterpart) ---------------------------------------------
 * A request loop over HBM-resident tables. `lanes` worker threads each own a context
 * (CUDA stream + scratch memory); a free lane takes the queued requests in arrival order,
 * up to max_batch, while their predicted device footprint fits in memory_budget minus what
 * running batches hold, and runs them as one gpudb_batch_run. Requests that arrive while
 * other batches are on the GPU are admitted by the next free lane, so work of different
 * batches overlaps on the device. max_batch = 1 and lanes = 1 is the plain
 * one-query-at-a-time form. */
typedef struct gpudb_server gpudb_server;
typedef struct gpudb_serve_config {
  int32_t device;
  uint32_t lanes;            /* worker lanes (contexts), 1..16 */
  uint32_t max_batch;        /* requests per batch, >= 1 */
  uint32_t heavy_lanes;      /* 0: every lane takes every request; else the last heavy_lanes lanes
                                take only Q6/Q1 requests over more than 2^24 rows and the others
                                the rest (a long scan never holds up short requests); must be
                                below `lanes` */
  uint64_t memory_budget;    /* bytes of predicted device footprint admitted at once; 0 = no limit */
} gpudb_serve_config;
typedef struct gpudb_serve_stats {
  uint64_t submitted, completed, failed, batches, max_batch_seen;
  uint64_t peak_admitted_bytes;
} gpudb_serve_stats;

int gpudb_serve_open(const gpudb_serve_config* cfg, gpudb_server** out);
/* Queues a request (caller-owned until it completes). GPUDB_E_BUSY if its predicted
 * footprint alone exceeds the budget, GPUDB_E_CLOSED after close. */
int gpudb_serve_submit(gpudb_server* s, gpudb_request* req, uint64_t* ticket);
/* Waits up to timeout_ms for a ticket; returns the request's status (GPUDB_E_TIMEOUT if it
 * is still running) and its submit-to-completion latency in milliseconds. */
int gpudb_serve_wait(gpudb_server* s, uint64_t ticket, double timeout_ms, double* latency_ms);
int gpudb_serve_stats_get(gpudb_server* s, gpudb_serve_stats* out);
/* Runs `reqs` once on every lane (lanes in parallel, each a synchronous batch) so that
 * the lanes' scratch memory is sized before traffic arrives; results are written to the
 * requests' outputs. Call it before submitting; it returns the first failing status. */
int gpudb_serve_warmup(gpudb_server* s, gpudb_request* reqs, uint32_t n);
/* Predicted device footprint of a request, in bytes (the admission estimate). */
uint64_t gpudb_request_footprint(const gpudb_request* req);
/* Stops accepting requests, finishes the queued ones, and frees the lanes. */
int gpudb_serve_close(gpudb_server* s);

/* ---- merging shard results (the reference runs on one device and merges nothing; these
 *      combine the results of row shards, one per GPU or per call) ------------------------
 * Host-only and exact: they need no context and no GPU. Q6 and Q1 partials of disjoint row
 * ranges add (int64 / int128 sums); Q9 groups of disjoint fact rows add per (nation, year)
 * and come out ordered by nation asc, year desc; Q3 top-k lists merge into the top k of
 * their union when the shards hold disjoint sets of orders (lineitem split by order key, so
 * each order's revenue is complete in one shard). */
int gpudb_q6_result_merge(const gpudb_q6_result* parts, uint32_t n, gpudb_q6_result* out);
int gpudb_q1_result_merge(const gpudb_q1_result* parts, uint32_t n, gpudb_q1_result* out);
/* groups: the parts' groups back to back, counts[i] of part i; at most `capacity` groups
 * written, *n_out the total. */
int gpudb_q9_result_merge(const gpudb_q9_group* groups, const uint32_t* counts, uint32_t n,
                          gpudb_q9_group* out, uint32_t capacity, uint32_t* n_out);
int gpudb_q3_result_merge(const gpudb_q3_result* parts, uint32_t n, int32_t k, gpudb_q3_result* out);

#ifdef __cplusplus
}
#endif
#endif /* GPUDB_CAPI_H */
