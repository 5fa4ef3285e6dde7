// Caller written against the reference's OLAP-core signatures, built against
// the B200 library through include/olap_reference_api.hpp.  It builds a small
// star schema in host memory the way the reference's gen_data lays it out
// (int8 dimension vectors with DIM_NULL, keys in [0, size] inclusive, so the
// byte past each vector is read), calls the three OLAPcore entry points with
// the reference's argument lists, and checks the int total against a direct
// loop over the same arrays.  Prints "OK <total>" on success.
#define OLAP_B200_DROP_IN
#include "olap_reference_api.hpp"

#include <cstdio>
#include <vector>

static uint32_t lcg(uint64_t& s) {
  s = s * 6364136223846793005ull + 1442695040888963407ull;
  return static_cast<uint32_t>(s >> 33);
}

int main() {
  const int sizes[4] = {3000, 200, 20000, 2555};
  const double sele[4] = {0.5, 0.8, 0.3, 1.0};
  const int groups[4] = {5, 3, 7, 4};
  const int size_lineorder = 1000003;
  uint64_t seed = 42;
  std::vector<std::vector<int8_t>> dv(4);
  std::vector<std::vector<int32_t>> fk(4);
  for (int t = 0; t < 4; ++t) {
    dv[t].resize(sizes[t] + 1);
    for (int i = 0; i < sizes[t]; ++i)
      dv[t][i] = (lcg(seed) % 1000) < sele[t] * 1000 ? static_cast<int8_t>(lcg(seed) % groups[t]) : OLAP_DIM_NULL;
    dv[t][sizes[t]] = 0;  // the byte past the end that keys == size read
    fk[t].resize(size_lineorder);
    for (int i = 0; i < size_lineorder; ++i) fk[t][i] = static_cast<int32_t>(lcg(seed) % (sizes[t] + 1));
  }
  std::vector<int32_t> M1(size_lineorder), M2(size_lineorder);
  for (int i = 0; i < size_lineorder; ++i) {
    M1[i] = static_cast<int32_t>(lcg(seed) % 10000 + 1);
    M2[i] = static_cast<int32_t>(lcg(seed) % 10000 + 1);
  }
  int8_t* dimvec_array[4] = {dv[0].data(), dv[1].data(), dv[2].data(), dv[3].data()};
  int32_t* fk_array[4] = {fk[0].data(), fk[1].data(), fk[2].data(), fk[3].data()};
  int orders[4] = {2, 0, 1, 3};
  int factor[4] = {groups[0] * groups[1] * groups[3], groups[1] * groups[3], groups[3], 1};
  int dimvec_nums = 4;
  int group_nums = groups[0] * groups[1] * groups[2] * groups[3];
  int n = size_lineorder;

  // Direct loop with the reference's per-row contract.
  std::vector<uint32_t> gv(group_nums, 0);
  for (int r = 0; r < n; ++r) {
    int g = 0;
    bool ok = true;
    for (int j = 0; j < dimvec_nums && ok; ++j) {
      const int c = dimvec_array[orders[j]][fk_array[orders[j]][r]];
      if (c == OLAP_DIM_NULL) ok = false;
      else g += c * factor[j];
    }
    if (ok) gv[g] += M1[r] + M2[r];
  }
  int expect = 0;
  for (int g = 0; g < group_nums; ++g) expect += gv[g];

  const int a = OLAPcore_rowwise(dimvec_array, fk_array, orders, dimvec_nums, factor, n, group_nums,
                                 M1.data(), M2.data(), 48);
  const int b = OLAPcore_vwm_dv(dimvec_array, fk_array, orders, dimvec_nums, factor, n, group_nums,
                                M1.data(), M2.data(), 48);
  const int c = OLAPcore_vwm_sv(dimvec_array, fk_array, orders, dimvec_nums, factor, n, group_nums,
                                M1.data(), M2.data(), 48);
  if (olap_b200::olap_last_status() != OLAP_OK) {
    std::printf("FAIL status %d\n", olap_b200::olap_last_status());
    return 1;
  }
  if (a != expect || b != expect || c != expect) {
    std::printf("FAIL %d %d %d expected %d\n", a, b, c, expect);
    return 1;
  }
  std::printf("OK %d %lld\n", a, static_cast<long long>(olap_b200::olap_last_total()));
  return 0;
}
