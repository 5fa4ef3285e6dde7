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
