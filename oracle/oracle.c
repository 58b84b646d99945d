/*
 * oracle.c -- CPU oracle (test infrastructure only; see oracle.h). Parity status: the
 * query logic is pinned against the reference's own kernels compiled for the CPU
 * (oracle/ref_harness.cpp) within float32 tolerance, since the reference computes in
 * float32; exact integer results are pinned against an independent big-integer Python
 * restatement (tests/golden/make_golden.py). The reference ships no golden vectors.
 */
#define _GNU_SOURCE
#include "oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>

typedef __int128 i128;
typedef unsigned __int128 u128;

/* ------------------------------------------------------------------------------------
 * Generator restatement: value(seed, stream, row) = F(K(seed, stream) + (row+1)*G) with
 * F the SplitMix64 output function, K(seed, s) = F(seed*G + (s+1)*0xD1B54A32D192ED03),
 * G = 0x9E3779B97F4A7C15, and uniform(lo, hi) = lo + floor(value * (hi-lo+1) / 2^64).
 * ------------------------------------------------------------------------------------ */
static uint64_t mix64(uint64_t x) {
  x ^= x >> 30; x *= 0xBF58476D1CE4E5B9ull;
  x ^= x >> 27; x *= 0x94D049BB133111EBull;
  x ^= x >> 31;
  return x;
}
static const uint64_t G = 0x9E3779B97F4A7C15ull;
static uint64_t stream_of(uint64_t seed, uint32_t s) { return mix64(seed * G + (uint64_t)(s + 1) * 0xD1B54A32D192ED03ull); }
static int64_t unif(uint64_t key, uint64_t row, int64_t lo, int64_t hi) {
  uint64_t v = mix64(key + (row + 1) * G);
  uint64_t span = (uint64_t)(hi - lo + 1);
  return lo + (int64_t)(uint64_t)(((u128)v * span) >> 64);
}

/* random stream ids (table*16 + column) */
enum { S_SHIP = 16, S_QTY, S_PRICE, S_DISC, S_TAX, S_FLAG, S_STATUS, S_OPICK, S_PART, S_SSLOT, S_RUN,
       S_COMMIT, S_RECEIPT, S_MODE,
       S_SEG = 32, S_CNATION, S_OCUST = 48, S_ODATE, S_OPRIO, S_OCOMMENT, S_PFLAG = 64, S_PTYPE, S_NATION = 80, S_COST = 96 };

/* order comment: n = U[2,9] words (sub-draw r*16), word i = U[0,23] (sub-draw r*16+1+i) of the
 * vocabulary below, joined by single spaces, stopping at the first word that would pass 79
 * characters; NUL-padded to 80 bytes */
static const char* const VOCAB[24] = {
  "special", "requests", "packages", "deposits", "accounts", "instructions", "foxes", "ideas", "theodolites",
  "pinto", "beans", "platelets", "furiously", "carefully", "quickly", "slyly", "blithely", "regular", "final",
  "pending", "ironic", "express", "bold", "even"};
static void comment_of(uint64_t key, uint64_t r, char* out) {
  int n = 0;
  const int words = (int)unif(key, r * 16, 2, 9);
  for (int i = 0; i < words; i++) {
    const char* w = VOCAB[unif(key, r * 16 + 1 + i, 0, 23)];
    const int wl = (int)strlen(w);
    if (n + (n ? 1 : 0) + wl > 79) break;
    if (n) out[n++] = ' ';
    memcpy(out + n, w, (size_t)wl);
    n += wl;
  }
  memset(out + n, 0, (size_t)(80 - n));
}

static int32_t supp_of(int64_t part, int64_t j, int64_t n_supp) { return (int32_t)((part + j * (n_supp / 4)) % n_supp); }

int or_gen_column(const or_spec* sp, int32_t column, void* dst) {
  const uint64_t seed = sp->seed, off = sp->row_offset, n = sp->n_rows;
  int32_t* i32 = (int32_t*)dst; int64_t* i64 = (int64_t*)dst; uint8_t* u8 = (uint8_t*)dst;
  uint64_t i;
  switch (column) {
  case 1: { uint64_t k = stream_of(seed, S_SHIP); for (i = 0; i < n; i++) i32[i] = (int32_t)unif(k, off + i, 0, 2526); return 0; }
  case 2: { uint64_t k = stream_of(seed, S_QTY); for (i = 0; i < n; i++) i32[i] = (int32_t)unif(k, off + i, 1, 50); return 0; }
  case 3: { uint64_t kq = stream_of(seed, S_QTY), kp = stream_of(seed, S_PRICE);
            for (i = 0; i < n; i++) i64[i] = unif(kq, off + i, 1, 50) * unif(kp, off + i, 90000, 209900); return 0; }
  case 4: { uint64_t k = stream_of(seed, S_DISC); for (i = 0; i < n; i++) i32[i] = (int32_t)unif(k, off + i, 0, 10); return 0; }
  case 5: { uint64_t k = stream_of(seed, S_TAX); for (i = 0; i < n; i++) i32[i] = (int32_t)unif(k, off + i, 0, 8); return 0; }
  case 6: { uint64_t k = stream_of(seed, S_FLAG); for (i = 0; i < n; i++) u8[i] = (uint8_t)unif(k, off + i, 0, 2); return 0; }
  case 7: { uint64_t k = stream_of(seed, S_STATUS); for (i = 0; i < n; i++) u8[i] = (uint8_t)unif(k, off + i, 0, 1); return 0; }
  case 8:
    if (sp->n_orders <= 0) return -1;
    if (sp->order_mode == 2) {
      uint64_t k = stream_of(seed, S_OPICK);
      for (i = 0; i < n; i++) i32[i] = (int32_t)(4 * unif(k, off + i, 0, sp->n_orders - 1) + 1);
      return 0;
    } else if (sp->order_mode == 1) {
      /* runs of 1..7 rows; run s belongs to order s mod n_orders */
      uint64_t k = stream_of(seed, S_RUN), row = 0, s = 0, end = off + n;
      while (row < end) {
        int64_t len = unif(k, s, 1, 7);
        int32_t key = (int32_t)(4 * (int64_t)(s % (uint64_t)sp->n_orders) + 1);
        for (int64_t j = 0; j < len && row < end; j++, row++)
          if (row >= off) i32[row - off] = key;
        s++;
      }
      return 0;
    }
    return -1;
  case 9: { if (sp->n_parts <= 0) return -1; uint64_t k = stream_of(seed, S_PART);
            for (i = 0; i < n; i++) i32[i] = (int32_t)unif(k, off + i, 0, sp->n_parts - 1); return 0; }
  case 10: { if (sp->n_parts <= 0 || sp->n_supp < 4) return -1;
             uint64_t kp = stream_of(seed, S_PART), ks = stream_of(seed, S_SSLOT);
             for (i = 0; i < n; i++) i32[i] = supp_of(unif(kp, off + i, 0, sp->n_parts - 1), unif(ks, off + i, 0, 3), sp->n_supp);
             return 0; }
  /* commit = ship + [-91, 89], receipt = ship + [1, 30], mode 0..6, priority 1..5 */
  case 11: { uint64_t ks = stream_of(seed, S_SHIP), k = stream_of(seed, S_COMMIT);
             for (i = 0; i < n; i++) i32[i] = (int32_t)(unif(ks, off + i, 0, 2526) + unif(k, off + i, -91, 89)); return 0; }
  case 12: { uint64_t ks = stream_of(seed, S_SHIP), k = stream_of(seed, S_RECEIPT);
             for (i = 0; i < n; i++) i32[i] = (int32_t)(unif(ks, off + i, 0, 2526) + unif(k, off + i, 1, 30)); return 0; }
  case 13: { uint64_t k = stream_of(seed, S_MODE); for (i = 0; i < n; i++) u8[i] = (uint8_t)unif(k, off + i, 0, 6); return 0; }
  case 33: { uint64_t k = stream_of(seed, S_OPRIO); for (i = 0; i < n; i++) u8[i] = (uint8_t)unif(k, off + i, 1, 5); return 0; }
  case 34: { uint64_t k = stream_of(seed, S_OCOMMENT); for (i = 0; i < n; i++) comment_of(k, off + i, (char*)u8 + i * 80); return 0; }
  case 20: case 30: case 40: case 50:
    for (i = 0; i < n; i++) i32[i] = (column == 30) ? (int32_t)(4 * (off + i) + 1) : (int32_t)(off + i);
    return 0;
  case 21: { uint64_t k = stream_of(seed, S_SEG); for (i = 0; i < n; i++) u8[i] = (uint8_t)unif(k, off + i, 0, 4); return 0; }
  case 22: { uint64_t k = stream_of(seed, S_CNATION); for (i = 0; i < n; i++) u8[i] = (uint8_t)unif(k, off + i, 0, 24); return 0; }
  case 31: { if (sp->n_cust <= 0) return -1; uint64_t k = stream_of(seed, S_OCUST);
             for (i = 0; i < n; i++) i32[i] = (int32_t)unif(k, off + i, 0, sp->n_cust - 1); return 0; }
  case 32: { uint64_t k = stream_of(seed, S_ODATE); for (i = 0; i < n; i++) i32[i] = (int32_t)unif(k, off + i, 0, 2405); return 0; }
  case 42: { uint64_t k = stream_of(seed, S_PTYPE); for (i = 0; i < n; i++) u8[i] = (uint8_t)unif(k, off + i, 0, 149); return 0; }
  case 41: { uint64_t k = stream_of(seed, S_PFLAG); for (i = 0; i < n; i++) u8[i] = unif(k, off + i, 0, 999) < 55; return 0; }
  case 51: { uint64_t k = stream_of(seed, S_NATION); for (i = 0; i < n; i++) u8[i] = (uint8_t)unif(k, off + i, 0, 24); return 0; }
  case 60: for (i = 0; i < n; i++) i32[i] = (int32_t)((off + i) / 4); return 0;
  case 61: if (sp->n_supp < 4) return -1;
           for (i = 0; i < n; i++) i32[i] = supp_of((int64_t)((off + i) / 4), (int64_t)((off + i) % 4), sp->n_supp);
           return 0;
  case 62: { uint64_t k = stream_of(seed, S_COST); for (i = 0; i < n; i++) i64[i] = unif(k, off + i, 100, 100000); return 0; }
  default: return -1;
  }
}

/* ---- Q6: predicate and measure of kernels/q6.metal:36-44 (short-circuit &&), exact ---- */
void or_q6(uint64_t n, const int32_t* ship, const int32_t* disc, const int32_t* qty,
           const int64_t* ext, int32_t lo, int32_t hi, int32_t dlo, int32_t dhi, int32_t qlt,
           int64_t* revenue, uint64_t* matched) {
  int64_t rev = 0; uint64_t m = 0;
  for (uint64_t i = 0; i < n; i++) {
    if (ship[i] >= lo && ship[i] < hi && disc[i] >= dlo && disc[i] <= dhi && qty[i] < qlt) {
      rev += ext[i] * (int64_t)disc[i];
      m++;
    }
  }
  *revenue = rev; *matched = m;
}

/* ---- Q1: filter and binning of kernels/q1.metal:73-94 (bin = flag*2 + status), with the
 *      measures exact instead of rounded per row ---------------------------------------- */
static void put128(uint64_t* dst, i128 v) { dst[0] = (uint64_t)(u128)v; dst[1] = (uint64_t)((u128)v >> 64); }

typedef struct q1acc { uint64_t cnt; i128 qty, base, disc, charge, dsum; } q1acc;

static void q1_range(uint64_t b, uint64_t e, const int32_t* ship, const int32_t* qty, const int64_t* ext,
                     const int32_t* disc, const int32_t* tax, const uint8_t* flag, const uint8_t* status,
                     int32_t ship_le, q1acc* acc) {
  for (uint64_t i = b; i < e; i++) {
    if (ship[i] > ship_le) continue;
    if (flag[i] > 2 || status[i] > 1) continue;
    q1acc* a = &acc[flag[i] * 2 + status[i]];
    i128 dp = (i128)ext[i] * (100 - disc[i]);
    a->cnt++;
    a->qty += qty[i];
    a->base += ext[i];
    a->disc += dp;
    a->charge += dp * (100 + tax[i]);
    a->dsum += disc[i];
  }
}

static void q1_emit(const q1acc* acc, uint64_t* out) {
  for (int g = 0; g < 6; g++) {
    uint64_t* o = out + g * 11;
    o[0] = acc[g].cnt;
    put128(o + 1, acc[g].qty); put128(o + 3, acc[g].base); put128(o + 5, acc[g].disc);
    put128(o + 7, acc[g].charge); put128(o + 9, acc[g].dsum);
  }
}

void or_q1(uint64_t n, const int32_t* ship, const int32_t* qty, const int64_t* ext,
           const int32_t* disc, const int32_t* tax, const uint8_t* flag, const uint8_t* status,
           int32_t ship_le, uint64_t* out) {
  q1acc acc[6]; memset(acc, 0, sizeof acc);
  q1_range(0, n, ship, qty, ext, disc, tax, flag, status, ship_le, acc);
  q1_emit(acc, out);
}

/* ---- threaded drivers for the timed CPU baseline --------------------------------------- */
typedef struct mt_job {
  uint64_t b, e; const int32_t *ship, *qty, *disc, *tax; const int64_t* ext;
  const uint8_t *flag, *status; int32_t a0, a1, a2, a3, a4;
  int64_t rev; uint64_t matched; q1acc acc[6];
} mt_job;

static void* q6_worker(void* p) {
  mt_job* j = (mt_job*)p;
  or_q6(j->e - j->b, j->ship + j->b, j->disc + j->b, j->qty + j->b, j->ext + j->b,
        j->a0, j->a1, j->a2, j->a3, j->a4, &j->rev, &j->matched);
  return NULL;
}
static void* q1_worker(void* p) {
  mt_job* j = (mt_job*)p;
  memset(j->acc, 0, sizeof j->acc);
  q1_range(j->b, j->e, j->ship, j->qty, j->ext, j->disc, j->tax, j->flag, j->status, j->a0, j->acc);
  return NULL;
}

static void run_jobs(int threads, uint64_t n, mt_job* base, void* (*fn)(void*), mt_job** out_jobs) {
  if (threads < 1) threads = 1;
  mt_job* jobs = (mt_job*)calloc((size_t)threads, sizeof(mt_job));
  pthread_t* th = (pthread_t*)calloc((size_t)threads, sizeof(pthread_t));
  for (int t = 0; t < threads; t++) {
    jobs[t] = *base;
    jobs[t].b = n * (uint64_t)t / (uint64_t)threads;
    jobs[t].e = n * (uint64_t)(t + 1) / (uint64_t)threads;
    pthread_create(&th[t], NULL, fn, &jobs[t]);
  }
  for (int t = 0; t < threads; t++) pthread_join(th[t], NULL);
  free(th);
  *out_jobs = jobs;
}

void or_q6_mt(int threads, uint64_t n, const int32_t* ship, const int32_t* disc,
              const int32_t* qty, const int64_t* ext, int32_t lo, int32_t hi, int32_t dlo,
              int32_t dhi, int32_t qlt, int64_t* revenue, uint64_t* matched) {
  mt_job base; memset(&base, 0, sizeof base);
  base.ship = ship; base.disc = disc; base.qty = qty; base.ext = ext;
  base.a0 = lo; base.a1 = hi; base.a2 = dlo; base.a3 = dhi; base.a4 = qlt;
  mt_job* jobs; if (threads < 1) threads = 1;
  run_jobs(threads, n, &base, q6_worker, &jobs);
  int64_t r = 0; uint64_t m = 0;
  for (int t = 0; t < threads; t++) { r += jobs[t].rev; m += jobs[t].matched; }
  free(jobs);
  *revenue = r; *matched = m;
}

void or_q1_mt(int threads, uint64_t n, const int32_t* ship, const int32_t* qty,
              const int64_t* ext, const int32_t* disc, const int32_t* tax,
              const uint8_t* flag, const uint8_t* status, int32_t ship_le, uint64_t* out) {
  mt_job base; memset(&base, 0, sizeof base);
  base.ship = ship; base.qty = qty; base.ext = ext; base.disc = disc; base.tax = tax;
  base.flag = flag; base.status = status; base.a0 = ship_le;
  mt_job* jobs; if (threads < 1) threads = 1;
  run_jobs(threads, n, &base, q1_worker, &jobs);
  q1acc acc[6]; memset(acc, 0, sizeof acc);
  for (int t = 0; t < threads; t++)
    for (int g = 0; g < 6; g++) {
      acc[g].cnt += jobs[t].acc[g].cnt; acc[g].qty += jobs[t].acc[g].qty;
      acc[g].base += jobs[t].acc[g].base; acc[g].disc += jobs[t].acc[g].disc;
      acc[g].charge += jobs[t].acc[g].charge; acc[g].dsum += jobs[t].acc[g].dsum;
    }
  free(jobs);
  q1_emit(acc, out);
}

/* ---- Q3: customer bitmap (kernels/q3.metal:43-55), orders filter + map
 *      (kernels/q3.metal:59-78), probe + per-order revenue (kernels/q3.metal:145-211),
 *      top-k order of sortAndPrintQ3 (src/infra.h:544-564) plus order_key as the last key -- */
typedef struct q3grp { int32_t key, date; int64_t rev; } q3grp;

static int q3_cmp(const void* a, const void* b) {
  const q3grp* x = (const q3grp*)a; const q3grp* y = (const q3grp*)b;
  if (x->rev != y->rev) return x->rev > y->rev ? -1 : 1;
  if (x->date != y->date) return x->date < y->date ? -1 : 1;
  if (x->key != y->key) return x->key < y->key ? -1 : 1;
  return 0;
}

uint64_t or_q3(uint64_t n_cu, const int32_t* cu_key, const uint8_t* cu_seg, int32_t cu_key_max,
               uint64_t n_or, const int32_t* or_key, const int32_t* or_cust,
               const int32_t* or_date, int32_t or_key_max,
               uint64_t n_li, const int32_t* li_order, const int32_t* li_ship,
               const int64_t* li_ext, const int32_t* li_disc,
               int32_t segment, int32_t date_lt, int32_t ship_gt, int32_t k,
               int32_t* top_key, int32_t* top_date, int64_t* top_rev) {
  uint8_t* cust_ok = (uint8_t*)calloc((size_t)cu_key_max + 1, 1);
  for (uint64_t i = 0; i < n_cu; i++)
    if (cu_seg[i] == segment) cust_ok[cu_key[i]] = 1;
  int64_t* order_row = (int64_t*)malloc(((size_t)or_key_max + 1) * sizeof(int64_t));
  for (int64_t i = 0; i <= or_key_max; i++) order_row[i] = -1;
  for (uint64_t i = 0; i < n_or; i++)
    if (or_date[i] < date_lt && or_cust[i] >= 0 && or_cust[i] <= cu_key_max && cust_ok[or_cust[i]])
      order_row[or_key[i]] = (int64_t)i;
  int64_t* rev = (int64_t*)calloc(n_or ? n_or : 1, sizeof(int64_t));
  uint8_t* hit = (uint8_t*)calloc(n_or ? n_or : 1, 1);
  for (uint64_t i = 0; i < n_li; i++) {
    if (li_ship[i] <= ship_gt) continue;
    int32_t key = li_order[i];
    if (key < 0 || key > or_key_max) continue;
    int64_t r = order_row[key];
    if (r < 0) continue;
    rev[r] += li_ext[i] * (int64_t)(100 - li_disc[i]);
    hit[r] = 1;
  }
  uint64_t groups = 0;
  for (uint64_t i = 0; i < n_or; i++) groups += hit[i];
  q3grp* g = (q3grp*)malloc((groups ? groups : 1) * sizeof(q3grp));
  uint64_t m = 0;
  for (uint64_t i = 0; i < n_or; i++)
    if (hit[i]) { g[m].key = or_key[i]; g[m].date = or_date[i]; g[m].rev = rev[i]; m++; }
  qsort(g, groups, sizeof(q3grp), q3_cmp);
  for (uint64_t i = 0; i < groups && i < (uint64_t)k; i++) {
    top_key[i] = g[i].key; top_date[i] = g[i].date; top_rev[i] = g[i].rev;
  }
  free(g); free(hit); free(rev); free(order_row); free(cust_ok);
  return groups;
}

/* ---- Q9: part filter (kernels/q9.metal:44-88, a flag column here), supplier -> nation
 *      (kernels/q9.metal:91-104), partsupp (part, supp) -> cost (kernels/q9.metal:109-162),
 *      orders -> year (kernels/q9.metal:165-189), probe chain and (nation<<16 | year)
 *      grouping (kernels/q9.metal:223-288), order of postProcessQ9 (src/infra.h:756-759) -- */
typedef struct kv64 { uint64_t key; int64_t val; uint8_t used; } kv64;

static uint64_t slot_of(uint64_t key, uint64_t mask) { return mix64(key) & mask; }

typedef struct q9grp { int32_t nation, year; int64_t profit; } q9grp;
static int q9_cmp(const void* a, const void* b) {
  const q9grp* x = (const q9grp*)a; const q9grp* y = (const q9grp*)b;
  if (x->nation != y->nation) return x->nation < y->nation ? -1 : 1;
  if (x->year != y->year) return x->year > y->year ? -1 : 1;
  return 0;
}

uint32_t or_q9(uint64_t n_pa, const int32_t* pa_key, const uint8_t* pa_flag, int32_t pa_key_max,
               uint64_t n_su, const int32_t* su_key, const uint8_t* su_nation, int32_t su_key_max,
               uint64_t n_ps, const int32_t* ps_part, const int32_t* ps_supp, const int64_t* ps_cost,
               uint64_t n_or, const int32_t* or_key, const int32_t* or_date, int32_t or_key_max,
               uint64_t n_li, const int32_t* li_part, const int32_t* li_supp, const int32_t* li_order,
               const int64_t* li_ext, const int32_t* li_disc, const int32_t* li_qty,
               uint32_t cap, int32_t* g_nation, int32_t* g_year, int64_t* g_profit) {
  uint8_t* part_ok = (uint8_t*)calloc((size_t)pa_key_max + 1, 1);
  for (uint64_t i = 0; i < n_pa; i++) if (pa_flag[i]) part_ok[pa_key[i]] = 1;
  int32_t* nation = (int32_t*)malloc(((size_t)su_key_max + 1) * sizeof(int32_t));
  for (int64_t i = 0; i <= su_key_max; i++) nation[i] = -1;
  for (uint64_t i = 0; i < n_su; i++) nation[su_key[i]] = su_nation[i];
  /* (part, supp) -> cost, open addressing */
  uint64_t cap_ps = 16; while (cap_ps < 2 * n_ps + 2) cap_ps <<= 1;
  kv64* ps = (kv64*)calloc(cap_ps, sizeof(kv64));
  for (uint64_t i = 0; i < n_ps; i++) {
    if (ps_part[i] < 0 || ps_part[i] > pa_key_max || !part_ok[ps_part[i]]) continue;
    uint64_t key = ((uint64_t)(uint32_t)ps_part[i] << 32) | (uint32_t)ps_supp[i];
    uint64_t s = slot_of(key, cap_ps - 1);
    while (ps[s].used && ps[s].key != key) s = (s + 1) & (cap_ps - 1);
    ps[s].used = 1; ps[s].key = key; ps[s].val = ps_cost[i];
  }
  int32_t* year = (int32_t*)malloc(((size_t)or_key_max + 1) * sizeof(int32_t));
  for (int64_t i = 0; i <= or_key_max; i++) year[i] = -1;
  for (uint64_t i = 0; i < n_or; i++) year[or_key[i]] = 1992 + or_date[i] / 365;
  uint64_t cap_g = 1u << 16;
  kv64* grp = (kv64*)calloc(cap_g, sizeof(kv64));
  uint32_t ngroups = 0;
  for (uint64_t i = 0; i < n_li; i++) {
    int32_t p = li_part[i];
    if (p < 0 || p > pa_key_max || !part_ok[p]) continue;
    int32_t s = li_supp[i];
    if (s < 0 || s > su_key_max || nation[s] < 0) continue;
    uint64_t key = ((uint64_t)(uint32_t)p << 32) | (uint32_t)s;
    uint64_t h = slot_of(key, cap_ps - 1);
    while (ps[h].used && ps[h].key != key) h = (h + 1) & (cap_ps - 1);
    if (!ps[h].used) continue;
    int32_t o = li_order[i];
    if (o < 0 || o > or_key_max || year[o] < 0) continue;
    int64_t profit = li_ext[i] * (int64_t)(100 - li_disc[i]) - ps[h].val * (int64_t)li_qty[i] * 100;
    uint64_t gk = ((uint64_t)(uint32_t)nation[s] << 16) | (uint32_t)year[o];
    uint64_t g = slot_of(gk, cap_g - 1);
    while (grp[g].used && grp[g].key != gk) g = (g + 1) & (cap_g - 1);
    if (!grp[g].used) { grp[g].used = 1; grp[g].key = gk; ngroups++; }
    grp[g].val += profit;
  }
  q9grp* out = (q9grp*)malloc((ngroups ? ngroups : 1) * sizeof(q9grp));
  uint32_t m = 0;
  for (uint64_t g = 0; g < cap_g; g++)
    if (grp[g].used) { out[m].nation = (int32_t)(grp[g].key >> 16); out[m].year = (int32_t)(grp[g].key & 0xFFFF); out[m].profit = grp[g].val; m++; }
  qsort(out, ngroups, sizeof(q9grp), q9_cmp);
  for (uint32_t i = 0; i < ngroups && i < cap; i++) { g_nation[i] = out[i].nation; g_year[i] = out[i].year; g_profit[i] = out[i].profit; }
  free(out); free(grp); free(year); free(ps); free(nation); free(part_ok);
  return ngroups;
}

/* ---- microbenchmarks: selection (kernels/microbenchmarks.metal:160-171), sum
 *      (:178-220), join count (:225-294), radix partition (:15-99), pairs (:104-156) ---- */
/* ---- Q4: kernels/q4.metal:21-37 (late bitmap) and :40-72 (date window, bitmap, bins) ---- */
void or_q4(uint64_t n_or, const int32_t* o_key, const int32_t* o_date, const uint8_t* o_prio, int32_t or_key_max,
           uint64_t n_li, const int32_t* l_key, const int32_t* l_commit, const int32_t* l_receipt, int32_t date_lo,
           int32_t date_hi, uint64_t* count5) {
  uint64_t i;
  uint8_t* late = or_key_max >= 0 ? (uint8_t*)calloc((size_t)or_key_max + 1, 1) : NULL;
  for (int b = 0; b < 5; b++) count5[b] = 0;
  if (!late) return;
  for (i = 0; i < n_li; i++)
    if (l_commit[i] < l_receipt[i] && l_key[i] >= 0 && l_key[i] <= or_key_max) late[l_key[i]] = 1;
  for (i = 0; i < n_or; i++) {
    if (o_date[i] < date_lo || o_date[i] >= date_hi) continue;
    if (o_key[i] < 0 || o_key[i] > or_key_max || !late[o_key[i]]) continue;
    if (o_prio[i] >= 1 && o_prio[i] <= 5) count5[o_prio[i] - 1]++;
  }
  free(late);
}

/* ---- Q12: kernels/q12.metal:87-99 (priority bitmap) and :22-66 (filters, 4 bins) ---- */
void or_q12(uint64_t n_or, const int32_t* o_key, const uint8_t* o_prio, int32_t or_key_max, uint64_t n_li,
            const int32_t* l_key, const int32_t* l_ship, const int32_t* l_commit, const int32_t* l_receipt,
            const uint8_t* l_mode, int32_t receipt_lo, int32_t receipt_hi, int32_t mode0, int32_t mode1,
            int32_t high_max, uint64_t* out4) {
  uint64_t i;
  uint8_t* high = or_key_max >= 0 ? (uint8_t*)calloc((size_t)or_key_max + 1, 1) : NULL;
  for (int b = 0; b < 4; b++) out4[b] = 0;
  if (high)
    for (i = 0; i < n_or; i++)
      if (o_prio[i] >= 1 && o_prio[i] <= high_max && o_key[i] >= 0 && o_key[i] <= or_key_max) high[o_key[i]] = 1;
  for (i = 0; i < n_li; i++) {
    const int m = l_mode[i] == mode0 ? 0 : (l_mode[i] == mode1 ? 1 : -1);
    if (m < 0) continue;
    const int32_t rd = l_receipt[i];
    if (rd < receipt_lo || rd >= receipt_hi) continue;
    if (l_commit[i] >= rd) continue;
    if (l_ship[i] >= l_commit[i]) continue;
    const int h = high && l_key[i] >= 0 && l_key[i] <= or_key_max && high[l_key[i]];
    out4[(h ? 0 : 2) + m]++;
  }
  free(high);
}

/* ---- Q5: kernels/q5.metal:19-125 (customer and supplier nation maps of the region, the
 * window's orders -> customer nation, lineitem rows whose supplier nation equals it) ---- */
void or_q5(uint64_t n_cu, const int32_t* cu_key, const uint8_t* cu_nation, int32_t cu_key_max, uint64_t n_su,
           const int32_t* su_key, const uint8_t* su_nation, int32_t su_key_max, uint64_t n_or, const int32_t* o_key,
           const int32_t* o_cust, const int32_t* o_date, int32_t or_key_max, uint64_t n_li, const int32_t* l_key,
           const int32_t* l_supp, const int64_t* l_ext, const int32_t* l_disc, int32_t date_lo, int32_t date_hi,
           uint32_t nation_mask, int64_t* revenue25) {
  uint64_t i;
  for (int n = 0; n < 25; n++) revenue25[n] = 0;
  if (cu_key_max < 0 || su_key_max < 0 || or_key_max < 0) return;
  uint8_t* cn = (uint8_t*)malloc((size_t)cu_key_max + 1);
  uint8_t* sn = (uint8_t*)malloc((size_t)su_key_max + 1);
  uint8_t* on = (uint8_t*)malloc((size_t)or_key_max + 1);
  memset(cn, 0xFF, (size_t)cu_key_max + 1);
  memset(sn, 0xFF, (size_t)su_key_max + 1);
  memset(on, 0xFF, (size_t)or_key_max + 1);
  for (i = 0; i < n_cu; i++) if (cu_nation[i] < 25 && (nation_mask >> cu_nation[i] & 1)) cn[cu_key[i]] = cu_nation[i];
  for (i = 0; i < n_su; i++) if (su_nation[i] < 25 && (nation_mask >> su_nation[i] & 1)) sn[su_key[i]] = su_nation[i];
  for (i = 0; i < n_or; i++) {
    if (o_date[i] < date_lo || o_date[i] >= date_hi) continue;
    if (o_cust[i] < 0 || o_cust[i] > cu_key_max) continue;
    on[o_key[i]] = cn[o_cust[i]];
  }
  for (i = 0; i < n_li; i++) {
    if (l_key[i] < 0 || l_key[i] > or_key_max || l_supp[i] < 0 || l_supp[i] > su_key_max) continue;
    const uint8_t n = on[l_key[i]];
    if (n == 0xFF || sn[l_supp[i]] != n) continue;
    revenue25[n] += l_ext[i] * (int64_t)(100 - l_disc[i]);
  }
  free(cn); free(sn); free(on);
}

/* calendar year of a day number (0 = 1992-01-01) */
static int year_len(int y) { return ((y % 4 == 0 && y % 100 != 0) || y % 400 == 0) ? 366 : 365; }
static int year_of_day(int32_t d) {
  int y = 1992;
  while (d < 0) { y--; d += year_len(y); }
  while (d >= year_len(y)) { d -= year_len(y); y++; }
  return y;
}
static uint8_t* nation_bytes(uint64_t n, const int32_t* key, const uint8_t* nation, int32_t key_max, uint32_t mask) {
  uint8_t* m = (uint8_t*)malloc((size_t)key_max + 1);
  memset(m, 0xFF, (size_t)key_max + 1);
  for (uint64_t i = 0; i < n; i++) if (nation[i] < 25 && (mask >> nation[i] & 1)) m[key[i]] = nation[i];
  return m;
}

/* ---- Q7: kernels/q7.metal:12-109 (supplier and customer maps of the two nations, orders ->
 * customer, lineitem in the ship window, pair and calendar year bins) ---- */
int or_q7(uint64_t n_cu, const int32_t* cu_key, const uint8_t* cu_nation, int32_t cu_key_max, uint64_t n_su,
          const int32_t* su_key, const uint8_t* su_nation, int32_t su_key_max, uint64_t n_or, const int32_t* o_key,
          const int32_t* o_cust, int32_t or_key_max, uint64_t n_li, const int32_t* l_key, const int32_t* l_supp,
          const int32_t* l_ship, const int64_t* l_ext, const int32_t* l_disc, int32_t a, int32_t b, int32_t ship_lo,
          int32_t ship_hi, int64_t* rev16, int32_t* first_year, int32_t* n_years) {
  uint64_t i;
  for (int j = 0; j < 16; j++) rev16[j] = 0;
  const int fy = year_of_day(ship_lo), ny = year_of_day(ship_hi) - fy + 1;
  *first_year = fy;
  *n_years = ny;
  if (ny < 1 || ny > 8) return -1;
  if (cu_key_max < 0 || su_key_max < 0 || or_key_max < 0) return 0;
  const uint32_t mask = (1u << a) | (1u << b);
  uint8_t* cn = nation_bytes(n_cu, cu_key, cu_nation, cu_key_max, mask);
  uint8_t* sn = nation_bytes(n_su, su_key, su_nation, su_key_max, mask);
  uint8_t* on = (uint8_t*)malloc((size_t)or_key_max + 1);
  memset(on, 0xFF, (size_t)or_key_max + 1);
  for (i = 0; i < n_or; i++) if (o_cust[i] >= 0 && o_cust[i] <= cu_key_max) on[o_key[i]] = cn[o_cust[i]];
  for (i = 0; i < n_li; i++) {
    if (l_ship[i] < ship_lo || l_ship[i] > ship_hi) continue;
    if (l_key[i] < 0 || l_key[i] > or_key_max || l_supp[i] < 0 || l_supp[i] > su_key_max) continue;
    const int c = on[l_key[i]], s = sn[l_supp[i]];
    const int pair = (s == a && c == b) ? 0 : (s == b && c == a) ? 1 : -1;
    if (pair < 0) continue;
    rev16[pair * 8 + year_of_day(l_ship[i]) - fy] += l_ext[i] * (int64_t)(100 - l_disc[i]);
  }
  free(cn); free(sn); free(on);
  return 0;
}

/* ---- Q8: kernels/q8.metal:9-76 (orders of the window with a customer of the region ->
 * order year, lineitem of the part type: total and the nation's share per year) ---- */
int or_q8(uint64_t n_cu, const int32_t* cu_key, const uint8_t* cu_nation, int32_t cu_key_max, uint64_t n_su,
          const int32_t* su_key, const uint8_t* su_nation, int32_t su_key_max, uint64_t n_pa, const int32_t* pa_key,
          const uint8_t* pa_type, int32_t pa_key_max, uint64_t n_or, const int32_t* o_key, const int32_t* o_cust,
          const int32_t* o_date, int32_t or_key_max, uint64_t n_li, const int32_t* l_key, const int32_t* l_part,
          const int32_t* l_supp, const int64_t* l_ext, const int32_t* l_disc, int32_t date_lo, int32_t date_hi,
          uint32_t region_mask, int32_t nation, int32_t part_type, int64_t* vol8, int64_t* nvol8, int32_t* first_year,
          int32_t* n_years) {
  uint64_t i;
  for (int j = 0; j < 8; j++) vol8[j] = nvol8[j] = 0;
  const int fy = year_of_day(date_lo), ny = year_of_day(date_hi) - fy + 1;
  *first_year = fy;
  *n_years = ny;
  if (ny < 1 || ny > 8) return -1;
  if (cu_key_max < 0 || su_key_max < 0 || pa_key_max < 0 || or_key_max < 0) return 0;
  uint8_t* cn = nation_bytes(n_cu, cu_key, cu_nation, cu_key_max, region_mask);
  uint8_t* sn = nation_bytes(n_su, su_key, su_nation, su_key_max, 1u << nation);
  uint8_t* pt = (uint8_t*)calloc((size_t)pa_key_max + 1, 1);
  uint8_t* oy = (uint8_t*)malloc((size_t)or_key_max + 1);
  memset(oy, 0xFF, (size_t)or_key_max + 1);
  for (i = 0; i < n_pa; i++) if (pa_type[i] == part_type) pt[pa_key[i]] = 1;
  for (i = 0; i < n_or; i++) {
    if (o_date[i] < date_lo || o_date[i] > date_hi) continue;
    if (o_cust[i] < 0 || o_cust[i] > cu_key_max || cn[o_cust[i]] == 0xFF) continue;
    oy[o_key[i]] = (uint8_t)(year_of_day(o_date[i]) - fy);
  }
  for (i = 0; i < n_li; i++) {
    if (l_part[i] < 0 || l_part[i] > pa_key_max || !pt[l_part[i]]) continue;
    if (l_key[i] < 0 || l_key[i] > or_key_max || oy[l_key[i]] == 0xFF) continue;
    if (l_supp[i] < 0 || l_supp[i] > su_key_max) continue;
    const int64_t r = l_ext[i] * (int64_t)(100 - l_disc[i]);
    vol8[oy[l_key[i]]] += r;
    if (sn[l_supp[i]] != 0xFF) nvol8[oy[l_key[i]]] += r;
  }
  free(cn); free(sn); free(pt); free(oy);
  return 0;
}

/* ---- Q10: kernels/q10.metal:8-54 (window map, returned rows), src/q10.cpp:102-121 (top-k) ---- */
typedef struct { int64_t rev; int32_t key; } q10row;
static int q10_cmp(const void* a, const void* b) {
  const q10row *x = (const q10row*)a, *y = (const q10row*)b;
  if (x->rev != y->rev) return x->rev > y->rev ? -1 : 1;
  return x->key < y->key ? -1 : (x->key > y->key);
}
uint64_t or_q10(uint64_t n_cu, const int32_t* cu_key, int32_t cu_key_max, uint64_t n_or, const int32_t* o_key,
                const int32_t* o_cust, const int32_t* o_date, int32_t or_key_max, uint64_t n_li, const int32_t* l_key,
                const uint8_t* l_flag, const int64_t* l_ext, const int32_t* l_disc, int32_t date_lo, int32_t date_hi,
                int32_t k, int32_t* top_key, int64_t* top_rev, int64_t* rev_out) {
  uint64_t i;
  if (cu_key_max < 0) return 0;
  uint8_t* is_cust = (uint8_t*)calloc((size_t)cu_key_max + 1, 1);
  int64_t* rev = (int64_t*)calloc((size_t)cu_key_max + 1, 8);
  int32_t* cust_of = or_key_max >= 0 ? (int32_t*)malloc(((size_t)or_key_max + 1) * 4) : NULL;
  for (i = 0; i < n_cu; i++) is_cust[cu_key[i]] = 1;
  if (cust_of) {
    for (i = 0; i <= (uint64_t)or_key_max; i++) cust_of[i] = -1;
    for (i = 0; i < n_or; i++)
      if (o_date[i] >= date_lo && o_date[i] < date_hi) cust_of[o_key[i]] = o_cust[i];
    for (i = 0; i < n_li; i++) {
      if (l_flag[i] != 2 || l_key[i] < 0 || l_key[i] > or_key_max) continue;
      const int32_t c = cust_of[l_key[i]];
      if (c < 0 || c > cu_key_max || !is_cust[c]) continue;
      rev[c] += l_ext[i] * (int64_t)(100 - l_disc[i]);
    }
  }
  q10row* rows = (q10row*)malloc(((size_t)cu_key_max + 1) * sizeof(q10row));
  uint64_t n = 0;
  for (int64_t c = 0; c <= cu_key_max; c++)
    if (rev[c] > 0) { rows[n].rev = rev[c]; rows[n].key = (int32_t)c; n++; }
  qsort(rows, n, sizeof(q10row), q10_cmp);
  for (int32_t r = 0; r < k; r++) {
    top_key[r] = r < (int64_t)n ? rows[r].key : -1;
    top_rev[r] = r < (int64_t)n ? rows[r].rev : 0;
  }
  if (rev_out) memcpy(rev_out, rev, ((size_t)cu_key_max + 1) * 8);
  free(is_cust); free(rev); free(cust_of); free(rows);
  return n;
}

/* ---- Q13: kernels/q13.metal:33-68 (first w1, then w2 after it), :110-127 (counts),
 * :133-168 (histogram), src/infra.h:783-800 (custdist desc, c_count desc) ---- */
static int like2(const char* s, const char* w1, const char* w2) {
  char buf[81];
  memcpy(buf, s, 80);
  buf[80] = 0;
  const char* a = strstr(buf, w1);
  return a && strstr(a + strlen(w1), w2) != NULL;
}
typedef struct { uint32_t c, d; } q13row;
static int q13_cmp(const void* a, const void* b) {
  const q13row *x = (const q13row*)a, *y = (const q13row*)b;
  if (x->d != y->d) return x->d > y->d ? -1 : 1;
  return x->c > y->c ? -1 : (x->c < y->c);
}
uint32_t or_q13(uint64_t n_cu, const int32_t* cu_key, int32_t cu_key_max, uint64_t n_or, const int32_t* o_cust,
                const char* o_comment, const char* w1, const char* w2, uint32_t* c_count, uint32_t* custdist,
                uint32_t cap) {
  uint64_t i;
  if (cu_key_max < 0 || n_cu == 0) return 0;
  uint32_t* cnt = (uint32_t*)calloc((size_t)cu_key_max + 1, 4);
  uint32_t top = 0;
  for (i = 0; i < n_or; i++)
    if (o_cust[i] >= 0 && o_cust[i] <= cu_key_max && !like2(o_comment + 80 * i, w1, w2)) cnt[o_cust[i]]++;
  for (i = 0; i < n_cu; i++) if (cnt[cu_key[i]] > top) top = cnt[cu_key[i]];
  uint32_t* hist = (uint32_t*)calloc((size_t)top + 1, 4);
  for (i = 0; i < n_cu; i++) hist[cnt[cu_key[i]]]++;
  q13row* rows = (q13row*)malloc(((size_t)top + 1) * sizeof(q13row));
  uint32_t n = 0;
  for (uint32_t c = 0; c <= top; c++) if (hist[c]) { rows[n].c = c; rows[n].d = hist[c]; n++; }
  qsort(rows, n, sizeof(q13row), q13_cmp);
  for (uint32_t r = 0; r < n && r < cap; r++) { c_count[r] = rows[r].c; custdist[r] = rows[r].d; }
  free(cnt); free(hist); free(rows);
  return n;
}

uint64_t or_select_lt(uint64_t n, const int32_t* col, int32_t value, uint32_t* bits, uint32_t* rows) {
  uint64_t c = 0;
  if (bits) memset(bits, 0, ((n + 31) / 32) * sizeof(uint32_t));
  for (uint64_t i = 0; i < n; i++)
    if (col[i] < value) {
      if (bits) bits[i / 32] |= 1u << (i % 32);
      if (rows) rows[c] = (uint32_t)i;
      c++;
    }
  return c;
}

int64_t or_sum_i32(uint64_t n, const int32_t* col) {
  int64_t s = 0;
  for (uint64_t i = 0; i < n; i++) s += col[i];
  return s;
}

static int cmp_i32(const void* a, const void* b) {
  int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
  return x < y ? -1 : x > y;
}

uint64_t or_join_count(uint64_t nb, const int32_t* bkeys, uint64_t np, const int32_t* pkeys) {
  int32_t* s = (int32_t*)malloc((nb ? nb : 1) * sizeof(int32_t));
  memcpy(s, bkeys, nb * sizeof(int32_t));
  qsort(s, nb, sizeof(int32_t), cmp_i32);
  uint64_t c = 0;
  for (uint64_t i = 0; i < np; i++)
    if (nb && bsearch(&pkeys[i], s, nb, sizeof(int32_t), cmp_i32)) c++;
  free(s);
  return c;
}

uint32_t or_key_hash(int32_t key) {
  uint32_t h = (uint32_t)key;
  h ^= h >> 16; h *= 0x45d9f3bu; h ^= h >> 16;
  return h;
}

void or_radix_histogram(uint64_t n, const int32_t* keys, int32_t bits, uint32_t* hist) {
  uint32_t parts = 1u << bits;
  memset(hist, 0, parts * sizeof(uint32_t));
  for (uint64_t i = 0; i < n; i++) hist[or_key_hash(keys[i]) & (parts - 1)]++;
}

void or_radix_partition(uint64_t n, const int32_t* keys, const int32_t* payload, int32_t bits,
                        int32_t* keys_out, int32_t* payload_out, uint32_t* offsets) {
  uint32_t parts = 1u << bits;
  uint32_t* hist = (uint32_t*)calloc(parts, sizeof(uint32_t));
  or_radix_histogram(n, keys, bits, hist);
  uint32_t run = 0;
  for (uint32_t p = 0; p < parts; p++) { offsets[p] = run; run += hist[p]; }
  offsets[parts] = run;
  uint32_t* cur = (uint32_t*)malloc(parts * sizeof(uint32_t));
  memcpy(cur, offsets, parts * sizeof(uint32_t));
  for (uint64_t i = 0; i < n; i++) {
    uint32_t p = or_key_hash(keys[i]) & (parts - 1);
    keys_out[cur[p]] = keys[i];
    if (payload && payload_out) payload_out[cur[p]] = payload[i];
    cur[p]++;
  }
  free(cur); free(hist);
}

typedef struct kidx { int32_t key; int32_t row; } kidx;
static int cmp_kidx(const void* a, const void* b) {
  const kidx* x = (const kidx*)a; const kidx* y = (const kidx*)b;
  if (x->key != y->key) return x->key < y->key ? -1 : 1;
  return x->row < y->row ? -1 : x->row > y->row;
}

uint64_t or_join_pairs(uint64_t nb, const int32_t* bkeys, uint64_t np, const int32_t* pkeys,
                       uint64_t cap, int32_t* out_b, int32_t* out_p) {
  kidx* s = (kidx*)malloc((nb ? nb : 1) * sizeof(kidx));
  for (uint64_t i = 0; i < nb; i++) { s[i].key = bkeys[i]; s[i].row = (int32_t)i; }
  qsort(s, nb, sizeof(kidx), cmp_kidx);
  uint64_t c = 0;
  for (uint64_t i = 0; i < np; i++) {
    /* lower bound of pkeys[i] */
    uint64_t lo = 0, hi = nb;
    while (lo < hi) { uint64_t mid = (lo + hi) / 2; if (s[mid].key < pkeys[i]) lo = mid + 1; else hi = mid; }
    for (uint64_t j = lo; j < nb && s[j].key == pkeys[i]; j++) {
      if (c < cap) { out_b[c] = s[j].row; out_p[c] = (int32_t)i; }
      c++;
    }
  }
  free(s);
  return c;
}
