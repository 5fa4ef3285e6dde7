// Caller written against the reference's operator signatures (code/join,
// select, project, group, aggregation, starjoin and the column-wise OLAP
// core), built against the B200 library through include/olap_reference_api.hpp.
// It declares the reference's structs the way include/metadata.h lays them
// out, fills host arrays, calls each operator with the reference's argument
// lists and checks every result against a direct loop over the same arrays
// (the reference's per-row contract).  Prints "OK <checks>" on success.
#define OLAP_B200_DROP_IN
#include "olap_reference_api.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <unordered_map>
#include <utility>
#include <vector>

typedef int idx;
typedef int T;
struct relation_t {  // include/metadata.h:263-270
  int32_t* key;
  int32_t* payload;
  uint64_t num_tuples;
  double payload_rate;
  int table_size;
};
struct row_store_min {  // include/metadata.h:251-256
  idx Ra;
  char Rb[52];
  idx Rc;
};
struct row_store_max {  // include/metadata.h:257-262
  idx Ra;
  char Rb[64];
  idx Rc;
};
struct fixed_arrays {  // include/metadata.h:245-250
  idx* pos_value1;
  idx* value2;
  idx array_size = 0;
};

static uint64_t g_seed = 7;
static uint32_t rnd() {
  g_seed = g_seed * 6364136223846793005ull + 1442695040888963407ull;
  return static_cast<uint32_t>(g_seed >> 33);
}
static int g_checks = 0;
#define CHECK(cond, what)                                                            \
  do {                                                                               \
    ++g_checks;                                                                      \
    if (!(cond)) {                                                                   \
      std::printf("FAIL %s (status %d)\n", what, olap_b200::olap_last_status());     \
      std::exit(1);                                                                  \
    }                                                                                \
  } while (0)

int main() {
  const int N = 1000003;
  // ---- join ----
  {
    const int nr = 1 << 16, ns = N;
    std::vector<int32_t> rk(nr), rp(nr), sk(ns), sp(ns, 1);
    for (int i = 0; i < nr; ++i) {
      rk[i] = static_cast<int32_t>(rnd() % (2 * nr));  // duplicates: the last row wins
      rp[i] = static_cast<int32_t>(rnd() % 2001) - 1000;
    }
    for (int i = 0; i < ns; ++i) sk[i] = static_cast<int32_t>(rnd() % (2 * nr));
    relation_t R{rk.data(), rp.data(), static_cast<uint64_t>(nr), 1.0, nr};
    relation_t S{sk.data(), sp.data(), static_cast<uint64_t>(ns), 1.0, ns};
    std::vector<int> vec(2 * nr, 0), want_vec(2 * nr, 0);
    for (int i = 0; i < nr; ++i) want_vec[rk[i]] = rp[i];
    build(&R, vec.data());
    CHECK(olap_b200::olap_last_status() == OLAP_OK && vec == want_vec, "vector build");
    int want = 0;
    for (int i = 0; i < ns; ++i) want += want_vec[sk[i]];
    CHECK(probe(&S, vec.data()) == want, "vector probe");
    CHECK(probe_prefetch(&S, vec.data()) == want, "vector probe_prefetch");
    std::unordered_map<int, int> ht;
    build(&R, ht);
    CHECK(olap_b200::olap_last_status() == OLAP_OK, "hash build");
    CHECK(probe(&S, ht) == want, "hash probe");
    // a map the caller filled itself is probed through its entries
    std::unordered_map<int, int> own;
    for (int i = 0; i < nr; ++i) own[rk[i]] = rp[i];
    CHECK(probe(&S, own) == want, "hash probe of a caller's map");
    olap_b200::release(ht);
    olap_b200::release(own);
  }
  // ---- select ----
  {
    std::vector<T> Ra(N), Rb(N), Rc(N), Rd(N);
    for (int i = 0; i < N; ++i) {
      Ra[i] = static_cast<T>(rnd() % 1000 + 1);
      Rb[i] = static_cast<T>(rnd() % 1000 + 1);
      Rc[i] = static_cast<T>(rnd() % 1000 + 1);
      Rd[i] = static_cast<T>(rnd() % 7);
    }
    T val = 400;
    std::vector<int> res(N), want;
    for (int i = 0; i < N; ++i)
      if (Ra[i] <= val) want.push_back(i);
    idx k = sel_lt_T_fsel_independent_val_branching(N, res.data(), Ra.data(), &val, nullptr);
    CHECK(k == static_cast<idx>(want.size()) && std::equal(want.begin(), want.end(), res.begin()), "fsel");
    // chained through the selection vector
    std::vector<int> res2(N), want2;
    T val2 = 600;
    for (int r : want)
      if (Rb[r] <= val2) want2.push_back(r);
    idx k2 = sel_lt_T_fsel_independent_val_non_branching(k, res2.data(), Rb.data(), &val2, res.data());
    CHECK(k2 == static_cast<idx>(want2.size()) && std::equal(want2.begin(), want2.end(), res2.begin()),
          "fsel with if_sv");
    idx cond = 500, s = 0;
    for (int i = 0; i < N; ++i)
      if (Ra[i] <= cond && Rb[i] <= cond && Rc[i] <= cond) s += Rd[i];
    CHECK(selalgo_rowwise(cond, N, Ra.data(), Rb.data(), Rc.data(), Rd.data()) == s, "selalgo_rowwise");
  }
  // ---- project ----
  {
    const int n = 300007;
    std::vector<row_store_min> rmin(n);
    std::vector<row_store_max> rmax(n);
    std::vector<int> Ra(n), Rc(n);
    for (int i = 0; i < n; ++i) {
      Ra[i] = static_cast<int>(rnd() % 1000 + 1);
      Rc[i] = static_cast<int>(rnd() % 1000 + 1);
      rmin[i].Ra = rmax[i].Ra = Ra[i];
      rmin[i].Rc = rmax[i].Rc = Rc[i];
      for (int b = 0; b < 52; ++b) rmin[i].Rb[b] = static_cast<char>(rnd());
      for (int b = 0; b < 64; ++b) rmax[i].Rb[b] = static_cast<char>(rnd());
    }
    const int cond = 300;
    std::vector<std::pair<int, int>> want;
    for (int i = 0; i < n; ++i)
      if (Ra[i] <= cond && Rc[i] <= cond) want.emplace_back(Ra[i], Rc[i]);
    std::vector<std::pair<int, int>> r1, r2, r3;
    CHECK(proalgo_rowwise(cond, n, rmin.data(), r1) == static_cast<int>(want.size()) && r1 == want,
          "proalgo_rowwise row_store_min");
    CHECK(proalgo_rowwise(cond, n, rmax.data(), r2) == static_cast<int>(want.size()) && r2 == want,
          "proalgo_rowwise row_store_max");
    std::vector<idx> a(n), c(n);
    fixed_arrays fa;
    fa.pos_value1 = a.data();
    fa.value2 = c.data();
    const int k = proalgo_rowwise(cond, n, rmax.data(), fa);
    bool same = k == static_cast<int>(want.size());
    for (int i = 0; same && i < k; ++i) same = a[i] == want[i].first && c[i] == want[i].second;
    CHECK(same, "proalgo_rowwise fixed_arrays");
    std::vector<int> pos1(n), pos2(n);
    CHECK(proalgo_cwm_lm_ifv(cond, n, Ra.data(), Rc.data(), pos1.data(), pos2.data(), r3) ==
                  static_cast<int>(want.size()) && r3 == want,
          "proalgo_cwm_lm_ifv");
    std::vector<idx> a2(n + 5), c2(n + 5);
    fixed_arrays fb;
    fb.pos_value1 = a2.data();
    fb.value2 = c2.data();
    const int k2 = proalgo_cwm_lm_ifv(cond, n, Ra.data(), Rc.data(), pos1.data(), pos2.data(), fb, 5);
    same = k2 == static_cast<int>(want.size());
    for (int i = 0; same && i < k2; ++i) same = a2[5 + i] == want[i].first && c2[5 + i] == want[i].second;
    CHECK(same, "proalgo_cwm_lm_ifv fixed_arrays");
  }
  // ---- group-by ----
  {
    const int G = 4096;
    std::vector<int> vi(N), m1(N), m2(N);
    for (int i = 0; i < N; ++i) {
      vi[i] = static_cast<int>(rnd() % G) + 1;
      m1[i] = static_cast<int>(rnd() % 10) + 1;
      m2[i] = static_cast<int>(rnd() % 10) + 1;
    }
    std::vector<int> gv(G, 3), want(G, 3);
    for (int i = 0; i < N; ++i) want[vi[i] - 1] += m1[i] + m2[i];
    int64_t wt = 0;
    for (int g = 0; g < G; ++g) wt += want[g];
    const size_t n = N;
    CHECK(vector_group(n, vi.data(), m1.data(), m2.data(), gv.data(), G) == wt && gv == want, "vector_group");
    std::unordered_map<int, int> hm, hw;
    for (int i = 0; i < N; ++i) hw[vi[i] - 1] += m1[i] + m2[i];
    int64_t ht = 0;
    for (size_t i = 0; i != hw.size(); ++i) ht += hw[static_cast<int>(i)];
    CHECK(hashtable_group(n, vi.data(), m1.data(), m2.data(), hm) == ht && hm == hw, "hashtable_group");
  }
  // ---- aggregation ----
  {
    const int n = 1 << 20;
    std::vector<double> tax(n), qty(n), price(n);
    for (int i = 0; i < n; ++i) {
      tax[i] = (rnd() % 9) / 100.0;
      qty[i] = rnd() % 50 + 1;
      price[i] = (rnd() % 100000) / 100.0;
    }
    double want = 0.0;
    for (int i = 0; i < n; ++i) want += (price[i] * qty[i]) * tax[i] + price[i] * qty[i];
    const double got = aggalgo_rowwise(n, tax.data(), qty.data(), price.data());
    CHECK(std::fabs(got - want) <= 1e-12 * std::fabs(want), "aggalgo_rowwise");
  }
  // ---- star-join operator and the column-wise OLAP core ----
  {
    const int sizes[4] = {3000, 200, 20000, 2556};
    const int groups[4] = {5, 3, 7, 4};
    std::vector<std::vector<int8_t>> dv(4);
    std::vector<std::vector<int32_t>> fk(4);
    for (int t = 0; t < 4; ++t) {
      dv[t].resize(sizes[t] + 1);
      for (int i = 0; i < sizes[t]; ++i)
        dv[t][i] = (rnd() % 10) < 6 ? static_cast<int8_t>(rnd() % groups[t]) : OLAP_DIM_NULL;
      dv[t][sizes[t]] = 0;  // keys reach size, as the reference's generator draws them
      fk[t].resize(N);
      for (int i = 0; i < N; ++i) fk[t][i] = static_cast<int32_t>(rnd() % (sizes[t] + 1));
    }
    std::vector<int32_t> M1(N), M2(N);
    for (int i = 0; i < N; ++i) {
      M1[i] = static_cast<int32_t>(rnd() % 10000 + 1);
      M2[i] = static_cast<int32_t>(rnd() % 10000 + 1);
    }
    int want_count = 0;
    for (int i = 0; i < N; ++i)
      want_count += dv[0][fk[0][i]] != OLAP_DIM_NULL && dv[1][fk[1][i]] != OLAP_DIM_NULL &&
                    dv[2][fk[2][i]] != OLAP_DIM_NULL && dv[3][fk[3][i]] != OLAP_DIM_NULL;
    CHECK(starjoinalgo_rowwise(N, dv[0].data(), dv[1].data(), dv[2].data(), dv[3].data(), fk[0].data(),
                               fk[1].data(), fk[2].data(), fk[3].data()) == want_count,
          "starjoinalgo_rowwise");
    int8_t* dimvec_array[4] = {dv[0].data(), dv[1].data(), dv[2].data(), dv[3].data()};
    int32_t* fk_array[4] = {fk[0].data(), fk[1].data(), fk[2].data(), fk[3].data()};
    int orders[4] = {2, 0, 1, 3};
    int factor[4] = {groups[0] * groups[1] * groups[3], groups[1] * groups[3], groups[3], 1};
    int nd = 4, n = N, G = groups[0] * groups[1] * groups[2] * groups[3];
    std::vector<int16_t> want_gid(N);
    std::vector<uint32_t> want_gv(G, 0);
    for (int i = 0; i < N; ++i) {
      int g = 0;
      bool live = true;
      for (int j = 0; j < nd && live; ++j) {
        const int c = dimvec_array[orders[j]][fk_array[orders[j]][i]];
        if (c == OLAP_DIM_NULL) live = false;
        else g += c * factor[j];
      }
      want_gid[i] = live ? static_cast<int16_t>(g) : static_cast<int16_t>(32767);
      if (live) want_gv[g] += M1[i] + M2[i];
    }
    int want_total = 0;
    for (int g = 0; g < G; ++g) want_total += want_gv[g];
    std::vector<int16_t> gid(N);
    join_cwm_sv(dimvec_array, fk_array, orders, nd, gid.data(), factor, n, 16);
    CHECK(olap_b200::olap_last_status() == OLAP_OK && gid == want_gid, "join_cwm_sv");
    CHECK(agg_cwm_sv(gid.data(), n, M1.data(), M2.data(), G, 16) == want_total, "agg_cwm_sv");
    const int nthreads = 7;
    std::vector<std::vector<int64_t>> oid(nthreads, std::vector<int64_t>(N));
    std::vector<std::vector<int16_t>> og(nthreads, std::vector<int16_t>(N));
    int64_t* OID[nthreads];
    int16_t* OG[nthreads];
    int index[nthreads];
    for (int j = 0; j < nthreads; ++j) {
      OID[j] = oid[j].data();
      OG[j] = og[j].data();
    }
    join_cwm_dv(dimvec_array, fk_array, orders, nd, OID, OG, factor, index, n, nthreads);
    bool same = olap_b200::olap_last_status() == OLAP_OK;
    const int per = N / nthreads;
    for (int j = 0; same && j < nthreads; ++j) {
      const int b = per * j, e = j == nthreads - 1 ? N : per * (j + 1);
      int k = 0;
      for (int i = b; i < e && same; ++i)
        if (want_gid[i] != 32767) {
          same = OID[j][k] == i && OG[j][k] == want_gid[i];
          ++k;
        }
      same = same && index[j] == k;
    }
    CHECK(same, "join_cwm_dv per-thread lists");
    CHECK(agg_cwm_dv(OID, OG, index, n, M1.data(), M2.data(), G, nthreads) == want_total, "agg_cwm_dv");
  }
  std::printf("OK %d\n", g_checks);
  return 0;
}
