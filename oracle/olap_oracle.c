/*
 * CPU oracle for the OLAP-core star-join and its operators.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py load this library, and only as the checker;
 * the product (libolapcore_b200.so) never links or calls it.
 *
 * Each function is a plain-C restatement of the reference's algorithm
 * (panjd123/memory_database; file:line cited per function) with two
 * deliberate changes: sums are int64 instead of uint32, and measures are read
 * at the row's own position.  Parity of this restatement is pinned by
 *   (1) the reference's published grand totals at SF=100 (GPU/plot/old.py),
 *       reproduced through oracle_gen_olapcore_compat below, and
 *   (2) the reference's own CPU functions compiled from its sources into
 *       oracle/_ref (see oracle/Makefile), compared per group in tests/.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define DIM_NULL 127     /* include/metadata.h:69 */
#define SIZE_V 1024      /* include/metadata.h:68 */

enum { AGG_M1_PLUS_M2 = 0, AGG_M1 = 1, AGG_M2 = 2, AGG_M1_TIMES_M2 = 3, AGG_COUNT = 4 };

static int64_t agg_value(int a, int32_t x, int32_t y) {
  switch (a) {
    case AGG_M1_PLUS_M2: return (int64_t)x + y;
    case AGG_M1: return x;
    case AGG_M2: return y;
    case AGG_M1_TIMES_M2: return (int64_t)x * y;
    default: return 1;
  }
}

/* Plan of the reference's main (code/OLAPcore/test_multi_compute_operator.cpp
 * :1964-1987): tables with groups > 0 participate in table order, then
 * sort_by_rate (:223-233) swaps orders[i], orders[j] when sele[i] > sele[j]
 * (sele indexed by position, as the reference does), group_nums is the
 * product of the groups, and factor[i] is the product of the later tables'
 * groups when table orders[i] is a bitmap table, else 1. */
int oracle_plan(const double* sele, const int* bitmap, const int* groups, int* orders,
                int* factor, int* dimvec_nums, int64_t* group_nums) {
  int n = 0;
  for (int t = 0; t < 4; t++) {
    factor[t] = 1;
    orders[t] = -1;
  }
  for (int t = 0; t < 4; t++)
    if (groups[t] != 0) orders[n++] = t;
  for (int i = 0; i < n; i++)
    for (int j = i + 1; j < n; j++)
      if (sele[i] > sele[j]) {
        int tmp = orders[i];
        orders[i] = orders[j];
        orders[j] = tmp;
      }
  int64_t g = 1;
  for (int i = 0; i < n; i++) {
    g *= groups[orders[i]];
    for (int j = i + 1; j < n; j++) {
      if (bitmap[orders[i]] == 0) break;
      factor[i] *= groups[orders[j]];
    }
  }
  *dimvec_nums = n;
  *group_nums = g;
  return 0;
}

/* Star-join + group-by SUM following OLAPcore_vwm_sv_thread
 * (code/OLAPcore/test_multi_compute_operator.cpp:509-568): the fact range is
 * cut into size_v-row vectors; for each vector a static group-id vector is
 * built one dimension at a time (first dimension assigns, later ones add or
 * null), then surviving rows add their aggregate.  Differences, by design:
 * group ids are int64 with a separate null flag (any group count), sums are
 * int64, and keys and group ids are range-checked instead of being read out
 * of bounds.  A row with a key outside [0, dim_len) is dropped; it is
 * counted in *range_errors when none of its in-range keys meets DIM_NULL
 * (a row that a filter drops anyway is not an error), a rule that gives the
 * same count whatever order the dimensions are probed in.  A surviving row
 * whose group id is outside [0, n_groups) is dropped and counted too. */
int oracle_starjoin(int nd, const int8_t* const* dimvec, const int64_t* dim_len,
                    const int32_t* const* fk, const int32_t* factor, int64_t row_begin,
                    int64_t row_end, const int32_t* m1, const int32_t* m2, int n_aggs,
                    const int32_t* agg, int64_t n_groups, int64_t* group_sums, int64_t* totals,
                    int64_t* range_errors) {
  int64_t gid[SIZE_V];
  unsigned char live[SIZE_V], oob[SIZE_V];
  int64_t errs = 0;
  if (group_sums) memset(group_sums, 0, sizeof(int64_t) * (size_t)(n_groups * n_aggs));
  for (int a = 0; a < n_aggs; a++) totals[a] = 0;
  for (int64_t v = row_begin; v < row_end; v += SIZE_V) {
    const int64_t len = (row_end - v) < SIZE_V ? (row_end - v) : SIZE_V;
    for (int64_t j = 0; j < len; j++) {
      gid[j] = 0;
      live[j] = 1;
      oob[j] = 0;
    }
    for (int d = 0; d < nd; d++) {
      for (int64_t j = 0; j < len; j++) {
        if (!live[j]) continue;
        const int32_t k = fk[d][v + j];
        if (k < 0 || (int64_t)k >= dim_len[d]) {
          oob[j] = 1;
          continue;
        }
        const int c = dimvec[d][k];
        if (c == DIM_NULL)
          live[j] = 0;
        else
          gid[j] += (int64_t)c * factor[d];
      }
    }
    for (int64_t j = 0; j < len; j++) {
      if (!live[j]) continue;
      if (oob[j]) {
        errs++;
        continue;
      }
      if (gid[j] < 0 || gid[j] >= n_groups) {
        errs++;
        continue;
      }
      const int32_t x = m1 ? m1[v + j] : 0, y = m2 ? m2[v + j] : 0;
      for (int a = 0; a < n_aggs; a++) {
        const int64_t val = agg_value(agg[a], x, y);
        totals[a] += val;
        if (group_sums) group_sums[(int64_t)a * n_groups + gid[j]] += val;
      }
    }
  }
  if (range_errors) *range_errors = errs;
  return 0;
}

/* oracle_starjoin over nthreads contiguous row ranges (cut at size_v
 * boundaries, as the reference's fan-out cuts its ranges per thread), each
 * with private group sums that are added up at the end: the same result,
 * for checking full-size tables in seconds. */
typedef struct {
  int nd;
  const int8_t* const* dimvec;
  const int64_t* dim_len;
  const int32_t* const* fk;
  const int32_t* factor;
  int64_t row_begin, row_end;
  const int32_t* m1;
  const int32_t* m2;
  int n_aggs;
  const int32_t* agg;
  int64_t n_groups;
  int64_t* group_sums; /* private, or NULL */
  int64_t totals[2];
  int64_t errs;
} starjoin_part_t;

static void* starjoin_part(void* arg) {
  starjoin_part_t* a = (starjoin_part_t*)arg;
  oracle_starjoin(a->nd, a->dimvec, a->dim_len, a->fk, a->factor, a->row_begin, a->row_end, a->m1, a->m2,
                  a->n_aggs, a->agg, a->n_groups, a->group_sums, a->totals, &a->errs);
  return NULL;
}

int oracle_starjoin_mt(int nthreads, int nd, const int8_t* const* dimvec, const int64_t* dim_len,
                       const int32_t* const* fk, const int32_t* factor, int64_t row_begin, int64_t row_end,
                       const int32_t* m1, const int32_t* m2, int n_aggs, const int32_t* agg, int64_t n_groups,
                       int64_t* group_sums, int64_t* totals, int64_t* range_errors) {
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 256) nthreads = 256;
  if (n_aggs < 1 || n_aggs > 2) return -1;
  starjoin_part_t part[256];
  pthread_t th[256];
  const int64_t rows = row_end - row_begin;
  const int64_t vecs = (rows + SIZE_V - 1) / SIZE_V;
  const size_t gbytes = sizeof(int64_t) * (size_t)(n_groups * n_aggs);
  int rc = 0;
  for (int t = 0; t < nthreads; t++) {
    starjoin_part_t* a = &part[t];
    a->nd = nd;
    a->dimvec = dimvec;
    a->dim_len = dim_len;
    a->fk = fk;
    a->factor = factor;
    a->row_begin = row_begin + vecs * t / nthreads * SIZE_V;
    a->row_end = t + 1 == nthreads ? row_end : row_begin + vecs * (t + 1) / nthreads * SIZE_V;
    if (a->row_begin > row_end) a->row_begin = row_end;
    if (a->row_end > row_end) a->row_end = row_end;
    a->m1 = m1;
    a->m2 = m2;
    a->n_aggs = n_aggs;
    a->agg = agg;
    a->n_groups = n_groups;
    a->group_sums = group_sums ? (int64_t*)malloc(gbytes) : NULL;
    if (group_sums && !a->group_sums) rc = -1;
  }
  int started = 0;
  if (rc == 0)
    for (; started < nthreads; started++)
      if (pthread_create(&th[started], NULL, starjoin_part, &part[started]) != 0) {
        rc = -1;
        break;
      }
  for (int t = 0; t < started; t++) pthread_join(th[t], NULL);
  if (rc == 0) {
    if (group_sums) memset(group_sums, 0, gbytes);
    int64_t errs = 0;
    for (int a = 0; a < n_aggs; a++) totals[a] = 0;
    for (int t = 0; t < nthreads; t++) {
      for (int a = 0; a < n_aggs; a++) totals[a] += part[t].totals[a];
      errs += part[t].errs;
      if (group_sums)
        for (int64_t i = 0; i < n_groups * n_aggs; i++) group_sums[i] += part[t].group_sums[i];
    }
    if (range_errors) *range_errors = errs;
  }
  for (int t = 0; t < nthreads; t++) free(part[t].group_sums);
  return rc;
}

/* size_of_table (include/gendata_util.hpp:152-166). */
static int size_of_table(int table, double sf) {
  switch (table) {
    case 0: return (int)(30000 * sf);
    case 1: return (int)(2000 * sf);
    case 2: return (int)(200000 * (double)(1 + log2(sf)));
    case 3: return 7 * 365;
    default: return (int)(6000000 * sf);
  }
}

int oracle_size_of_table(int table, double sf) { return size_of_table(table, sf); }

/* The C library's rand() on glibc, restated (the reference runs on glibc and
 * never seeds it, so its data are this stream from seed 1).  glibc's default
 * generator (random_r.c, TYPE_3) is the additive lagged-Fibonacci generator
 * r[i] = r[i-3] + r[i-31] (mod 2^32) over 34 seed words: r[0] = seed,
 * r[i] = 16807 * r[i-1] mod (2^31 - 1) for i = 1..30, r[31..33] = r[0..2];
 * the first 310 outputs are discarded and rand() returns r[i] >> 1.  The
 * stream is generated a block at a time, so 2.4 billion draws (an SF=100
 * table) take seconds instead of the minutes of 2.4 billion locked libc
 * calls.  tests/ check it against the libc rand() of the build host. */
#define GLIBC_RAND_BLOCK 8192
typedef struct {
  uint32_t r[GLIBC_RAND_BLOCK + 34];
  int pos; /* next output index into r[34 .. 34 + GLIBC_RAND_BLOCK) */
} glibc_rand_t;

static void glibc_rand_refill(glibc_rand_t* g) {
  uint32_t* r = g->r;
  for (int i = 34; i < GLIBC_RAND_BLOCK + 34; i++) r[i] = r[i - 31] + r[i - 3];
  g->pos = 34;
}

static void glibc_rand_seed(glibc_rand_t* g, uint32_t seed) {
  int32_t w[34];
  w[0] = (int32_t)(seed == 0 ? 1 : seed);
  for (int i = 1; i < 31; i++) {
    const int64_t v = (16807LL * w[i - 1]) % 2147483647LL;
    w[i] = (int32_t)(v < 0 ? v + 2147483647LL : v);
  }
  for (int i = 31; i < 34; i++) w[i] = w[i - 31];
  /* r[0..33] hold the 34 words before the first raw value r[34] */
  for (int i = 0; i < 34; i++) g->r[i] = (uint32_t)w[i];
  glibc_rand_refill(g);
  /* the generator discards its first 310 values */
  for (int k = 0; k < 310; k++) {
    if (g->pos == GLIBC_RAND_BLOCK + 34) {
      memmove(g->r, g->r + GLIBC_RAND_BLOCK, 34 * sizeof(uint32_t));
      glibc_rand_refill(g);
    }
    g->pos++;
  }
}

static inline int glibc_rand(glibc_rand_t* g) {
  if (g->pos == GLIBC_RAND_BLOCK + 34) {
    memmove(g->r, g->r + GLIBC_RAND_BLOCK, 34 * sizeof(uint32_t));
    glibc_rand_refill(g);
  }
  return (int)(g->r[g->pos++] >> 1);
}

/* The first n values of rand() after srand(seed), restated (for the tests
 * that pin the restatement to the C library). */
int oracle_glibc_rand_stream(uint32_t seed, int64_t n, int32_t* out) {
  glibc_rand_t* g = (glibc_rand_t*)malloc(sizeof(glibc_rand_t));
  if (!g) return -1;
  glibc_rand_seed(g, seed);
  for (int64_t i = 0; i < n; i++) out[i] = glibc_rand(g);
  free(g);
  return 0;
}

/* rand_x overloads (include/gendata_util.hpp:174-197) over that stream
 * (RAND_MAX = 2^31 - 1 on glibc). */
static double rand_unit(glibc_rand_t* g) {
  return 0.0 + (double)glibc_rand(g) / ((double)(2147483647 / (1.0 - 0.0)));
}
static int rand_range(glibc_rand_t* g, int lo, int hi) { return glibc_rand(g) % (hi - lo + 1) + lo; }

/* The reference's OLAPcore data generator (include/gendata_util.hpp:449-542),
 * driven by glibc's rand() stream (restated above) from its default seed 1
 * (the reference never calls srand on this path).  Tables in order customer, supplier, part, date:
 * entry i is NULL unless rand_x(0.0,1.0) <= sele, then a code rand_x(0,
 * groups-1) for bitmap tables or 0 otherwise.  Then per fact row four keys
 * rand_x(0, size) (inclusive of size) and M1 = M2 = 5.  dimvec[t] must hold
 * size+1 bytes: the extra byte is set to 0, which is what the reference reads
 * past the end (the published totals reproduce only with 0 there). */
int oracle_gen_olapcore_compat(double sf, const double* sele, const int* bitmap, const int* groups,
                               int8_t* const* dimvec, int32_t* const* fk, int32_t* m1, int32_t* m2) {
  int size[4];
  for (int t = 0; t < 4; t++) size[t] = size_of_table(t, sf);
  const int64_t n = size_of_table(4, sf);
  glibc_rand_t* g = (glibc_rand_t*)malloc(sizeof(glibc_rand_t));
  if (!g) return -1;
  glibc_rand_seed(g, 1);
  for (int t = 0; t < 4; t++) {
    for (int i = 0; i < size[t]; i++) {
      if (bitmap[t])
        dimvec[t][i] = rand_unit(g) <= sele[t] ? (int8_t)rand_range(g, 0, groups[t] - 1) : DIM_NULL;
      else
        dimvec[t][i] = rand_unit(g) <= sele[t] ? 0 : DIM_NULL;
    }
    dimvec[t][size[t]] = 0;
  }
  /* Per fact row four keys rand() % (size + 1), drawn a block of the stream
   * at a time; the remainder by a run-time divisor d is taken exactly as
   * ((2^64 / d + 1) * x mod 2^64) * d >> 64 (Lemire, Kaser and Kurz, "Faster
   * remainder by direct computation", 2019), valid for every 32-bit x. */
  uint64_t mul[4];
  for (int t = 0; t < 4; t++) mul[t] = UINT64_C(0xFFFFFFFFFFFFFFFF) / (uint64_t)(size[t] + 1) + 1;
  int64_t i = 0;
  while (i < n) {
    int avail = (GLIBC_RAND_BLOCK + 34 - g->pos) / 4;
    if (avail == 0) {
      /* the next row straddles a refill: draw it value by value */
      for (int t = 0; t < 4; t++) fk[t][i] = rand_range(g, 0, size[t]);
      i++;
      continue;
    }
    if ((int64_t)avail > n - i) avail = (int)(n - i);
    const uint32_t* r = g->r + g->pos;
    for (int k = 0; k < avail; k++, i++)
      for (int t = 0; t < 4; t++) {
        const uint64_t x = r[4 * k + t] >> 1, low = mul[t] * x;
        fk[t][i] = (int32_t)(((unsigned __int128)low * (uint64_t)(size[t] + 1)) >> 64);
      }
    g->pos += 4 * avail;
  }
  if (m1)
    for (int64_t j = 0; j < n; j++) m1[j] = 5;
  if (m2)
    for (int64_t j = 0; j < n; j++) m2[j] = 5;
  free(g);
  return 0;
}

/* ---- the benchmark's seeded columns, restated ------------------------------
 * The GPU library generates the benchmark tables in HBM with counter-based
 * generators (value i of stream s under seed k is a splitmix64 finaliser of
 * a Weyl sequence).  These are the same definitions on the host, so that the
 * CPU baseline gets bit-identical inputs without loading the GPU library;
 * tests/ check them against the library's own host generators. */
static inline uint64_t sm_mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * UINT64_C(0xBF58476D1CE4E5B9);
  z = (z ^ (z >> 27)) * UINT64_C(0x94D049BB133111EB);
  return z ^ (z >> 31);
}
static inline uint64_t sm_key(uint64_t seed, uint64_t stream) {
  return sm_mix64(seed ^ sm_mix64(stream + UINT64_C(0x632BE59BD9B4E019)));
}
static inline uint64_t sm_draw(uint64_t key, uint64_t i) {
  return sm_mix64(key + (i + 1) * UINT64_C(0x9E3779B97F4A7C15));
}

typedef struct {
  int kind; /* 0 uniform int32, 1 dimension vector, 2 zipf */
  void* out;
  int64_t b, e;
  uint64_t key;
  int32_t lo;
  uint64_t span;   /* uniform: hi - lo + 1 */
  uint64_t thresh; /* dimension vector: pass when (r >> 32) < thresh */
  uint32_t groups;
  const uint64_t* cdf;
  int64_t nk;
} gen_part_t;

static void* gen_part(void* arg) {
  gen_part_t* a = (gen_part_t*)arg;
  for (int64_t i = a->b; i < a->e; i++) {
    const uint64_t r = sm_draw(a->key, (uint64_t)i);
    if (a->kind == 0) {
      ((int32_t*)a->out)[i] = (int32_t)((int64_t)a->lo + (int64_t)(((r >> 32) * a->span) >> 32));
    } else if (a->kind == 1) {
      ((int8_t*)a->out)[i] =
          (r >> 32) >= a->thresh ? (int8_t)DIM_NULL : (int8_t)(((r & 0xffffffffu) * a->groups) >> 32);
    } else {
      const uint64_t u = r >> 11;
      int64_t lo = 0, hi = a->nk - 1;
      while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (u < a->cdf[mid]) hi = mid; else lo = mid + 1;
      }
      ((int32_t*)a->out)[i] = (int32_t)lo;
    }
  }
  return NULL;
}

static int gen_run(gen_part_t proto, int64_t n, int nthreads) {
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 256) nthreads = 256;
  if (n < (1 << 16)) nthreads = 1;
  gen_part_t part[256];
  pthread_t th[256];
  int started = 0;
  for (int t = 0; t < nthreads; t++) {
    part[t] = proto;
    part[t].b = n * t / nthreads;
    part[t].e = n * (t + 1) / nthreads;
  }
  for (; started < nthreads; started++)
    if (pthread_create(&th[started], NULL, gen_part, &part[started]) != 0) break;
  for (int t = started; t < nthreads; t++) gen_part(&part[t]);
  for (int t = 0; t < started; t++) pthread_join(th[t], NULL);
  return 0;
}

/* value i uniform in [lo, hi]: lo + ((draw >> 32) * (hi - lo + 1)) >> 32 */
int oracle_gen_uniform_i32(int32_t* out, int64_t n, uint64_t seed, uint64_t stream, int32_t lo, int32_t hi,
                           int nthreads) {
  if (n < 0 || hi < lo) return -1;
  gen_part_t g;
  memset(&g, 0, sizeof(g));
  g.kind = 0;
  g.out = out;
  g.key = sm_key(seed, stream);
  g.lo = lo;
  g.span = (uint64_t)((int64_t)hi - lo + 1);
  return gen_run(g, n, nthreads);
}

/* entry i: DIM_NULL unless (draw >> 32) < sele * 2^32, else the code
 * ((draw mod 2^32) * groups) >> 32 */
int oracle_gen_dimvec(int8_t* out, int64_t n, uint64_t seed, uint64_t stream, double sele, int32_t groups,
                      int nthreads) {
  if (n < 0 || groups < 1 || groups > 127) return -1;
  gen_part_t g;
  memset(&g, 0, sizeof(g));
  g.kind = 1;
  g.out = out;
  g.key = sm_key(seed, stream);
  g.thresh = !(sele > 0.0) ? 0 : sele >= 1.0 ? (UINT64_C(1) << 32) : (uint64_t)ldexp(sele, 32);
  g.groups = (uint32_t)groups;
  return gen_run(g, n, nthreads);
}

/* Zipf(s) over n_keys keys: the smallest k with (draw >> 11) < cdf[k], the
 * CDF of k^-s scaled to 2^53 (long double sums, strictly increasing). */
int oracle_gen_zipf_i32(int32_t* out, int64_t n, uint64_t seed, uint64_t stream, int64_t n_keys, double s,
                        int nthreads) {
  if (n < 0 || n_keys < 1 || n_keys > INT32_MAX || !(s >= 0.0)) return -1;
  long double* w = (long double*)malloc(sizeof(long double) * (size_t)n_keys);
  uint64_t* cdf = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n_keys);
  if (!w || !cdf) {
    free(w);
    free(cdf);
    return -1;
  }
  long double tot = 0;
  for (int64_t k = 0; k < n_keys; k++) {
    w[k] = powl((long double)(k + 1), -(long double)s);
    tot += w[k];
  }
  const long double scale = ldexpl(1.0L, 53);
  long double acc = 0;
  uint64_t prev = 0;
  for (int64_t k = 0; k < n_keys; k++) {
    acc += w[k];
    uint64_t c = (uint64_t)(acc / tot * scale);
    if (c <= prev) c = prev + 1;
    cdf[k] = c;
    prev = c;
  }
  cdf[n_keys - 1] = UINT64_C(1) << 53;
  if (n_keys > 1 && cdf[n_keys - 2] >= cdf[n_keys - 1]) cdf[n_keys - 2] = cdf[n_keys - 1] - 1;
  free(w);
  gen_part_t g;
  memset(&g, 0, sizeof(g));
  g.kind = 2;
  g.out = out;
  g.key = sm_key(seed, stream);
  g.cdf = cdf;
  g.nk = n_keys;
  const int rc = gen_run(g, n, nthreads);
  free(cdf);
  return rc;
}

/* ---- operators: select, project, join, group-by, aggregation ----------- */

enum { CMP_LE = 0, CMP_LT = 1 };
static int cmp_pass(int32_t v, int32_t val, int cmp) { return cmp == CMP_LT ? v < val : v <= val; }

/* sel_lt_T_fsel_independent_val_branching (select/test_select_option.cpp
 * :391-423): row ids (or entries of the input selection vector) that pass,
 * in order.  Input entries outside [0, col_len) are dropped and counted. */
int64_t oracle_select_rowids(const int32_t* col, int64_t col_len, int32_t val, int cmp,
                             const int32_t* in_rowids, int64_t n_in, int32_t* out,
                             int64_t* range_errors) {
  int64_t j = 0, errs = 0;
  if (!in_rowids) {
    for (int64_t i = 0; i < col_len; i++)
      if (cmp_pass(col[i], val, cmp)) out[j++] = (int32_t)i;
  } else {
    for (int64_t i = 0; i < n_in; i++) {
      const int32_t r = in_rowids[i];
      if (r < 0 || r >= col_len) { errs++; continue; }
      if (cmp_pass(col[r], val, cmp)) out[j++] = r;
    }
  }
  if (range_errors) *range_errors = errs;
  return j;
}

/* sel_lt_T_bmp_independent_val_branching (select:424-440), packed LSB first. */
void oracle_select_bitmap(const int32_t* col, int64_t n, int32_t val, int cmp, uint32_t* bits) {
  for (int64_t w = 0; w < (n + 31) / 32; w++) bits[w] = 0;
  for (int64_t i = 0; i < n; i++)
    if (cmp_pass(col[i], val, cmp)) bits[i >> 5] |= 1u << (i & 31);
}

/* selalgo_rowwise (select:450-467): SUM(Rd) over rows with Ra, Rb, Rc <= cond. */
int64_t oracle_selalgo(int32_t cond, int64_t n, const int32_t* ra, const int32_t* rb,
                       const int32_t* rc, const int32_t* rd, int64_t* count) {
  int64_t s = 0, c = 0;
  for (int64_t i = 0; i < n; i++)
    if (ra[i] <= cond && rb[i] <= cond && rc[i] <= cond) {
      s += rd[i];
      c++;
    }
  if (count) *count = c;
  return s;
}

/* proalgo_rowwise (project/test_project_option.cpp:34-49): pairs (Ra, Rc) of
 * the rows with Ra <= cond and Rc <= cond, in row order. */
int64_t oracle_project_pairs(int32_t cond, int64_t n, const int32_t* ra, const int32_t* rc,
                             int32_t* out_a, int32_t* out_c) {
  int64_t j = 0;
  for (int64_t i = 0; i < n; i++)
    if (ra[i] <= cond && rc[i] <= cond) {
      out_a[j] = ra[i];
      out_c[j] = rc[i];
      j++;
    }
  return j;
}

/* Late materialisation: outs[c][i] = cols[c][rowids[i]] (0 when out of range). */
int64_t oracle_gather(const int32_t* rowids, int64_t k, int ncols, const int32_t* const* cols,
                      int64_t col_len, int32_t* const* outs) {
  int64_t errs = 0;
  for (int64_t i = 0; i < k; i++) {
    const int32_t r = rowids[i];
    const int ok = r >= 0 && r < col_len;
    errs += !ok;
    for (int c = 0; c < ncols; c++) outs[c][i] = ok ? cols[c][r] : 0;
  }
  return errs;
}

/* build + probe of join/test_join_option.cpp: vector[key] = payload in row
 * order (:30-36, last row wins), then SUM vector[key] over the probe keys
 * (:58-64).  Build keys outside [0, len) and probe keys outside [0, len) are
 * counted in *range_errors and skipped.  vector must be zeroed (or hold the
 * caller's initial values). */
int64_t oracle_vecjoin(const int32_t* rk, const int32_t* rp, int64_t nr, const int32_t* sk, int64_t ns,
                       int32_t* vector, int64_t len, int64_t* range_errors) {
  int64_t errs = 0, s = 0;
  for (int64_t i = 0; i < nr; i++) {
    if (rk[i] < 0 || rk[i] >= len) { errs++; continue; }
    vector[rk[i]] = rp[i];
  }
  for (int64_t i = 0; i < ns; i++) {
    if (sk[i] < 0 || sk[i] >= len) { errs++; continue; }
    s += vector[sk[i]];
  }
  if (range_errors) *range_errors = errs;
  return s;
}

/* Hash join through a dictionary with the semantics of std::unordered_map
 * (join:44-50, :90-96): last build row wins per key, a missing probe key adds
 * 0.  Implemented with a private open-addressing table (keys INT32_MIN
 * skipped as in the library); also returns the match count and, when
 * out_rows is given, the matches (probe row, payload) in probe-row order. */
int64_t oracle_hashjoin(const int32_t* rk, const int32_t* rp, int64_t nr, const int32_t* sk, int64_t ns,
                        int64_t* matches, int32_t* out_rows, int32_t* out_payload) {
  int64_t cap = 16;
  while (cap < 2 * nr + 16) cap <<= 1;
  int32_t* keys = (int32_t*)malloc(sizeof(int32_t) * cap);
  int32_t* vals = (int32_t*)malloc(sizeof(int32_t) * cap);
  for (int64_t i = 0; i < cap; i++) keys[i] = INT32_MIN;
  for (int64_t i = 0; i < nr; i++) {
    const int32_t k = rk[i];
    if (k == INT32_MIN) continue;
    uint64_t h = ((uint64_t)(uint32_t)k * 2654435761u) & (cap - 1);
    while (keys[h] != INT32_MIN && keys[h] != k) h = (h + 1) & (cap - 1);
    keys[h] = k;
    vals[h] = rp[i];
  }
  int64_t s = 0, m = 0;
  for (int64_t i = 0; i < ns; i++) {
    const int32_t k = sk[i];
    if (k == INT32_MIN) continue;
    uint64_t h = ((uint64_t)(uint32_t)k * 2654435761u) & (cap - 1);
    while (keys[h] != INT32_MIN && keys[h] != k) h = (h + 1) & (cap - 1);
    if (keys[h] == k) {
      s += vals[h];
      if (out_rows) {
        out_rows[m] = (int32_t)i;
        out_payload[m] = vals[h];
      }
      m++;
    }
  }
  free(keys);
  free(vals);
  if (matches) *matches = m;
  return s;
}

/* oracle_hashjoin's sum and match count with the probe side cut over
 * nthreads threads (the build is the same sequential, last-row-wins
 * dictionary), for full-size probe sides. */
typedef struct {
  const int32_t* keys;
  const int32_t* vals;
  int64_t cap;
  const int32_t* sk;
  int64_t b, e;
  int64_t sum, matches;
} probe_part_t;

static void* probe_part(void* arg) {
  probe_part_t* a = (probe_part_t*)arg;
  int64_t s = 0, m = 0;
  for (int64_t i = a->b; i < a->e; i++) {
    const int32_t k = a->sk[i];
    if (k == INT32_MIN) continue;
    uint64_t h = ((uint64_t)(uint32_t)k * 2654435761u) & (a->cap - 1);
    while (a->keys[h] != INT32_MIN && a->keys[h] != k) h = (h + 1) & (a->cap - 1);
    if (a->keys[h] == k) {
      s += a->vals[h];
      m++;
    }
  }
  a->sum = s;
  a->matches = m;
  return NULL;
}

int64_t oracle_hashjoin_sum_mt(int nthreads, const int32_t* rk, const int32_t* rp, int64_t nr, const int32_t* sk,
                               int64_t ns, int64_t* matches) {
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 256) nthreads = 256;
  int64_t cap = 16;
  while (cap < 2 * nr + 16) cap <<= 1;
  int32_t* keys = (int32_t*)malloc(sizeof(int32_t) * cap);
  int32_t* vals = (int32_t*)malloc(sizeof(int32_t) * cap);
  if (!keys || !vals) {
    free(keys);
    free(vals);
    if (matches) *matches = -1;
    return 0;
  }
  for (int64_t i = 0; i < cap; i++) keys[i] = INT32_MIN;
  for (int64_t i = 0; i < nr; i++) {
    const int32_t k = rk[i];
    if (k == INT32_MIN) continue;
    uint64_t h = ((uint64_t)(uint32_t)k * 2654435761u) & (cap - 1);
    while (keys[h] != INT32_MIN && keys[h] != k) h = (h + 1) & (cap - 1);
    keys[h] = k;
    vals[h] = rp[i];
  }
  probe_part_t part[256];
  pthread_t th[256];
  int started = 0;
  for (int t = 0; t < nthreads; t++) {
    part[t] = (probe_part_t){keys, vals, cap, sk, ns * t / nthreads, ns * (t + 1) / nthreads, 0, 0};
  }
  for (; started < nthreads; started++)
    if (pthread_create(&th[started], NULL, probe_part, &part[started]) != 0) break;
  for (int t = started; t < nthreads; t++) probe_part(&part[t]); /* threads refused: run here */
  for (int t = 0; t < started; t++) pthread_join(th[t], NULL);
  int64_t s = 0, m = 0;
  for (int t = 0; t < nthreads; t++) {
    s += part[t].sum;
    m += part[t].matches;
  }
  free(keys);
  free(vals);
  if (matches) *matches = m;
  return s;
}

/* vector_group (group/test_group_option.cpp:44-60) with int64 sums: 1-based
 * group ids, returns the total; ids outside [1, G] counted and skipped. */
int64_t oracle_vector_group(int64_t n, const int32_t* idx, const int32_t* m1, const int32_t* m2, int64_t G,
                            int64_t* gv, int64_t* counts, int64_t* range_errors) {
  int64_t tot = 0, errs = 0;
  for (int64_t g = 0; g < G; g++) {
    gv[g] = 0;
    if (counts) counts[g] = 0;
  }
  for (int64_t i = 0; i < n; i++) {
    const int64_t g = (int64_t)idx[i] - 1;
    if (g < 0 || g >= G) { errs++; continue; }
    const int64_t v = (int64_t)m1[i] + m2[i];
    gv[g] += v;
    if (counts) counts[g]++;
    tot += v;
  }
  if (range_errors) *range_errors = errs;
  return tot;
}

/* aggalgo in int64 fixed point: SUM price*qty*(100 + tax_pct) (mod 2^64). */
int64_t oracle_agg_fixed(int64_t n, const int32_t* price, const int32_t* qty, const int32_t* tax) {
  uint64_t s = 0;
  for (int64_t i = 0; i < n; i++)
    s += (uint64_t)((int64_t)price[i] * qty[i]) * (uint64_t)((int64_t)100 + tax[i]);
  return (int64_t)s;
}

/* aggalgo_rowwise (aggregation/test_aggregation_option.cpp:28-37) in double. */
double oracle_agg_f64(int64_t n, const double* tax, const double* qty, const double* price) {
  double r = 0.0;
  for (int64_t i = 0; i < n; i++) r += (price[i] * qty[i]) * tax[i] + price[i] * qty[i];
  return r;
}

/* join_cwm_sv thread body (OLAPcore/test_multi_compute_operator.cpp:290-322)
 * over all dimensions: int16 group id or GROUP_NULL; keys outside [0, len)
 * give GROUP_NULL and are counted. */
int64_t oracle_join_cwm_sv(int nd, const int8_t* const* dimvec, const int64_t* len, const int32_t* const* fk,
                           const int32_t* factor, int64_t n, int16_t* gid) {
  int64_t errs = 0;
  for (int64_t r = 0; r < n; r++) {
    int ok = 1;
    for (int d = 0; d < nd; d++)
      if (fk[d][r] < 0 || fk[d][r] >= len[d]) ok = 0;
    if (!ok) { errs++; gid[r] = 32767; continue; }
    int32_t g = 0;
    for (int d = 0; d < nd && ok; d++) {
      const int c = dimvec[d][fk[d][r]];
      if (c == DIM_NULL) ok = 0;
      else g += c * factor[d];
    }
    gid[r] = ok ? (int16_t)g : (int16_t)32767;
  }
  return errs;
}

/* starjoinalgo_cwm_sv (starjoin/test_starjoin_option.cpp:66-121) over the
 * four tables in order customer, supplier, part, date; returns the count of
 * entries that are not GROUP_NULL. */
int64_t oracle_starjoin_cwm_sv(const int8_t* const* dimvec, const int64_t* len, const int32_t* const* fk,
                               int64_t n, int32_t* result) {
  static const int shift[4] = {12, 8, 4, 0};
  int64_t c = 0;
  for (int64_t r = 0; r < n; r++) {
    int ok = 1;
    for (int d = 0; d < 4; d++)
      if (fk[d][r] < 0 || fk[d][r] >= len[d]) ok = 0;
    int32_t g = 0;
    for (int d = 0; d < 4 && ok; d++) {
      const int v = dimvec[d][fk[d][r]];
      if (v == DIM_NULL) ok = 0;
      else g += v << shift[d];
    }
    result[r] = ok ? g : 32767;
    c += result[r] != 32767;
  }
  return c;
}

/* TPC-H Q5 chain (TPCH_Q5/Q5.cpp:913-978) in int64 fixed point:
 * nation_sums[n] = SUM price * (100 - discount) over lines whose supplier
 * nation (s_nationkey[suppkey-1]) is in a region with key `region` and equals
 * the nation of the order's customer (c_nationkey[custkey-1]), the order dated
 * in [date1, date2).  Invalid references are counted and skipped. */
int64_t oracle_q5(const int32_t* r_regionkey, int64_t n_region, const int32_t* n_regionkey, int64_t n_nation,
                  const int32_t* s_nationkey, int64_t n_supp, const int32_t* c_nationkey, int64_t n_cust,
                  const int32_t* o_custkey, const int32_t* o_orderdate, int64_t n_orders, const int32_t* l_orderkey,
                  const int32_t* l_suppkey, const int32_t* l_price, const int32_t* l_discount, int64_t n_lines,
                  int32_t region, int32_t date1, int32_t date2, int64_t* nation_sums) {
  int64_t errs = 0;
  unsigned char ok_nation[64] = {0};
  for (int64_t n = 0; n < n_nation && n < 64; n++) {
    const int32_t r = n_regionkey[n];
    ok_nation[n] = r >= 0 && r < n_region && r_regionkey[r] == region;
  }
  int8_t* ds = (int8_t*)malloc((size_t)(n_supp > 0 ? n_supp : 1));
  int8_t* dor = (int8_t*)malloc((size_t)(n_orders > 0 ? n_orders : 1));
  for (int64_t i = 0; i < n_supp; i++) {
    const int32_t n = s_nationkey[i];
    ds[i] = (n >= 0 && n < 64 && ok_nation[n]) ? (int8_t)n : -1;
  }
  for (int64_t i = 0; i < n_orders; i++) {
    dor[i] = -1;
    if (o_orderdate[i] >= date1 && o_orderdate[i] < date2) {
      const int32_t c = o_custkey[i];
      if (c < 1 || c > n_cust) { errs++; continue; }
      const int32_t n = c_nationkey[c - 1];
      if (n >= 0 && n < 64 && ok_nation[n]) dor[i] = (int8_t)n;
    }
  }
  for (int64_t n = 0; n < n_nation; n++) nation_sums[n] = 0;
  for (int64_t i = 0; i < n_lines; i++) {
    const int32_t sk = l_suppkey[i], ok = l_orderkey[i];
    if (sk < 1 || sk > n_supp || ok < 0 || ok >= n_orders) { errs++; continue; }
    const int ns = ds[sk - 1];
    if (ns < 0 || dor[ok] != ns) continue;
    nation_sums[ns] += (int64_t)l_price[i] * (100 - l_discount[i]);
  }
  free(ds);
  free(dor);
  return errs;
}
