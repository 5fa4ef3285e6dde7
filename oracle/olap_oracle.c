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
 * int64, and a row whose key is outside [0, dim_len) or whose group id is
 * outside [0, n_groups) is dropped and counted in *range_errors instead of
 * being read out of bounds. */
int oracle_starjoin(int nd, const int8_t* const* dimvec, const int64_t* dim_len,
                    const int32_t* const* fk, const int32_t* factor, int64_t row_begin,
                    int64_t row_end, const int32_t* m1, const int32_t* m2, int n_aggs,
                    const int32_t* agg, int64_t n_groups, int64_t* group_sums, int64_t* totals,
                    int64_t* range_errors) {
  int64_t gid[SIZE_V];
  unsigned char live[SIZE_V];
  int64_t errs = 0;
  if (group_sums) memset(group_sums, 0, sizeof(int64_t) * (size_t)(n_groups * n_aggs));
  for (int a = 0; a < n_aggs; a++) totals[a] = 0;
  for (int64_t v = row_begin; v < row_end; v += SIZE_V) {
    const int64_t len = (row_end - v) < SIZE_V ? (row_end - v) : SIZE_V;
    for (int64_t j = 0; j < len; j++) {
      gid[j] = 0;
      live[j] = 1;
      for (int d = 0; d < nd; d++) {
        const int32_t k = fk[d][v + j];
        if (k < 0 || (int64_t)k >= dim_len[d]) {
          live[j] = 0;
          errs++;
          break;
        }
      }
    }
    for (int d = 0; d < nd; d++) {
      for (int64_t j = 0; j < len; j++) {
        if (!live[j]) continue;
        const int c = dimvec[d][fk[d][v + j]];
        if (c == DIM_NULL)
          live[j] = 0;
        else
          gid[j] += (int64_t)c * factor[d];
      }
    }
    for (int64_t j = 0; j < len; j++) {
      if (!live[j]) continue;
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

/* rand_x overloads (include/gendata_util.hpp:174-197). */
static double rand_unit(void) { return 0.0 + (double)rand() / ((double)(RAND_MAX / (1.0 - 0.0))); }
static int rand_range(int lo, int hi) { return rand() % (hi - lo + 1) + lo; }

/* The reference's OLAPcore data generator (include/gendata_util.hpp:449-542),
 * driven by the C library's rand() from its default seed (the reference never
 * calls srand on this path).  Tables in order customer, supplier, part, date:
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
  srand(1);
  for (int t = 0; t < 4; t++) {
    for (int i = 0; i < size[t]; i++) {
      if (bitmap[t])
        dimvec[t][i] = rand_unit() <= sele[t] ? (int8_t)rand_range(0, groups[t] - 1) : DIM_NULL;
      else
        dimvec[t][i] = rand_unit() <= sele[t] ? 0 : DIM_NULL;
    }
    dimvec[t][size[t]] = 0;
  }
  for (int64_t i = 0; i < n; i++) {
    for (int t = 0; t < 4; t++) fk[t][i] = rand_range(0, size[t]);
    if (m1) m1[i] = 5;
    if (m2) m2[i] = 5;
  }
  return 0;
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
