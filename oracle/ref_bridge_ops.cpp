// C-linkage bridges over the reference's operator modules (select, join,
// group, aggregation, starjoin, project), one shared object per module.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file once per
// module with -DREF_MODULE_<NAME> and that module's directory on the include
// path, so the translation unit below is the reference's unmodified source,
// read in place (its main() renamed by -Dmain=ref_module_main).
#include <cstdint>
#include <unordered_map>
#include <vector>

#if defined(REF_MODULE_SELECT)
#include "test_select_option.cpp"
extern "C" {
// selalgo_rowwise (select/test_select_option.cpp:450-467).
int ref_selalgo_rowwise(int cond, int n, const int* Ra, const int* Rb, const int* Rc, const int* Rd) {
  return selalgo_rowwise(cond, n, Ra, Rb, Rc, Rd);
}
// sel_lt_T_fsel_independent_val_branching (:391-423); if_sv may be NULL.
int ref_sel_fsel_branching(int n, int* res, const int* col, int val, int* if_sv) {
  return sel_lt_T_fsel_independent_val_branching(n, res, col, &val, if_sv);
}
// sel_lt_T_fsel_independent_val_non_branching (:172-205).
int ref_sel_fsel_non_branching(int n, int* res, const int* col, int val, int* if_sv) {
  return sel_lt_T_fsel_independent_val_non_branching(n, res, col, &val, if_sv);
}
// sel_lt_T_bmp_independent_val_branching (:424-440), one byte per row out.
void ref_sel_bmp(int n, unsigned char* out, const int* col, int val) {
  std::vector<bool> bm(n);
  sel_lt_T_bmp_independent_val_branching(n, bm, col, &val);
  for (int i = 0; i < n; ++i) out[i] = bm[i];
}
}
#elif defined(REF_MODULE_JOIN)
#include "test_join_option.cpp"
extern "C" {
// build/probe with direct addressing (join/test_join_option.cpp:30-36, 58-64).
int ref_vecjoin(const int32_t* rk, const int32_t* rp, uint64_t nr, const int32_t* sk, uint64_t ns,
                int* vector) {
  relation_t R, S;
  R.key = const_cast<int32_t*>(rk); R.payload = const_cast<int32_t*>(rp); R.num_tuples = nr;
  S.key = const_cast<int32_t*>(sk); S.payload = nullptr; S.num_tuples = ns;
  build(&R, vector);
  return probe(&S, vector);
}
// build/probe through std::unordered_map (:44-50, 90-96).
int ref_hashjoin(const int32_t* rk, const int32_t* rp, uint64_t nr, const int32_t* sk, uint64_t ns) {
  relation_t R, S;
  R.key = const_cast<int32_t*>(rk); R.payload = const_cast<int32_t*>(rp); R.num_tuples = nr;
  S.key = const_cast<int32_t*>(sk); S.payload = nullptr; S.num_tuples = ns;
  std::unordered_map<int, int> ht;
  build(&R, ht);
  return probe(&S, ht);
}
}
#elif defined(REF_MODULE_GROUP)
#include "test_group_option.cpp"
extern "C" {
// vector_group (group/test_group_option.cpp:44-60); group_vector zeroed by the caller.
int64_t ref_vector_group(uint64_t n, const int* vecInx, const int* m1, const int* m2, int* group_vector,
                         int group_num) {
  const size_t sz = n;
  return vector_group(sz, vecInx, m1, m2, group_vector, group_num);
}
// hashtable_group (:71-88).
int64_t ref_hashtable_group(uint64_t n, const int* vecInx, const int* m1, const int* m2) {
  const size_t sz = n;
  std::unordered_map<int, int> ht;
  return hashtable_group(sz, vecInx, m1, m2, ht);
}
}
#elif defined(REF_MODULE_AGGREGATION)
#include "test_aggregation_option.cpp"
extern "C" {
// aggalgo_rowwise (aggregation/test_aggregation_option.cpp:28-37).
double ref_aggalgo_rowwise(int n, const double* tax, const double* qty, const double* price) {
  return aggalgo_rowwise(n, tax, qty, price);
}
}
#elif defined(REF_MODULE_STARJOIN)
#include "test_starjoin_option.cpp"
extern "C" {
// starjoinalgo_rowwise (starjoin/test_starjoin_option.cpp:37-50).
int ref_starjoin_rowwise(int n, const int8_t* dc, const int8_t* ds, const int8_t* dp, const int8_t* dd,
                         const int32_t* fc, const int32_t* fs, const int32_t* fp, const int32_t* fd) {
  return starjoinalgo_rowwise(n, dc, ds, dp, dd, fc, fs, fp, fd);
}
// starjoinalgo_cwm_sv (:66-121); result is zeroed by this wrapper first (the
// reference adds the first dimension's code to it).
int ref_starjoin_cwm_sv(int n, const int8_t* dc, const int8_t* ds, const int8_t* dp, const int8_t* dd,
                        const int32_t* fc, const int32_t* fs, const int32_t* fp, const int32_t* fd,
                        int* result) {
  for (int i = 0; i < n; ++i) result[i] = 0;
  return starjoinalgo_cwm_sv(n, dc, ds, dp, dd, fc, fs, fp, fd, result);
}
}
#elif defined(REF_MODULE_PROJECT)
#include "test_project_option.cpp"
extern "C" {
// proalgo_rowwise over the module's own row stores (project/test_project_option
// .cpp:62-90 and :120-147, the static row_min / row_max arrays it declares at
// :20-21): the columns are written into the rows' Ra and Rc fields first, the
// pairs come back as two int arrays.  which: 0 row_store_min, 1
// row_store_max; n at most 2^26 (the arrays' length).
int ref_proalgo_rowwise(int which, int cond, int n, const int* Ra, const int* Rc, int* out_a, int* out_c) {
  fixed_arrays res;
  res.pos_value1 = out_a;
  res.value2 = out_c;
  if (which == 0) {
    for (int i = 0; i < n; ++i) {
      row_min[i].Ra = Ra[i];
      row_min[i].Rc = Rc[i];
    }
    return proalgo_rowwise(cond, n, row_min, res);
  }
  for (int i = 0; i < n; ++i) {
    row_max[i].Ra = Ra[i];
    row_max[i].Rc = Rc[i];
  }
  return proalgo_rowwise(cond, n, row_max, res);
}
// proalgo_cwm_lm_ifv (:527-595), late materialisation over the columns.
int ref_proalgo_cwm_lm_ifv(int cond, int n, const int* Ra, const int* Rc, int* out_a, int* out_c) {
  std::vector<int> pos1(n > 0 ? n : 1), pos2(n > 0 ? n : 1);
  fixed_arrays res;
  res.pos_value1 = out_a;
  res.value2 = out_c;
  return proalgo_cwm_lm_ifv(cond, n, Ra, Rc, pos1.data(), pos2.data(), res, 0);
}
// proalgo_cwm_em (:190-232), early materialisation, with pre_size 0.
int ref_proalgo_cwm_em(int cond, int n, const int* Ra, const int* Rc, int* out_a, int* out_c) {
  fixed_arrays res;
  res.pos_value1 = out_a;
  res.value2 = out_c;
  return proalgo_cwm_em(cond, n, Ra, Rc, res, 0);
}
}
#endif
