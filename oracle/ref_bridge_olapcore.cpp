// C-linkage bridge over the reference's own OLAPcore translation unit.
//
// TEST INFRASTRUCTURE ONLY (see olap_oracle.c).  oracle/Makefile compiles
// this file with the reference's code/OLAPcore directory on the include path,
// so the translation unit below is the reference's unmodified source, read in
// place; its main() is renamed by -Dmain=ref_olapcore_main.  The wrappers let
// tests and the CPU baseline call the reference's fan-out functions (which
// return only the int grand total) and its per-thread bodies (which expose
// per-group sums) with caller-owned buffers.
#include "test_multi_compute_operator.cpp"

extern "C" {

// OLAPcore_rowwise (code/OLAPcore/test_multi_compute_operator.cpp:973).
int ref_OLAPcore_rowwise(int8_t** dimvec_array, int32_t** fk_array, int* orders, int dimvec_nums,
                         int* factor, int size_lineorder, int group_nums, int32_t* M1, int32_t* M2,
                         int nthreads) {
  return OLAPcore_rowwise(dimvec_array, fk_array, orders, dimvec_nums, factor, size_lineorder,
                          group_nums, M1, M2, nthreads);
}

// OLAPcore_vwm_dv (:1052).
int ref_OLAPcore_vwm_dv(int8_t** dimvec_array, int32_t** fk_array, int* orders, int dimvec_nums,
                        int* factor, int size_lineorder, int group_nums, int32_t* M1, int32_t* M2,
                        int nthreads) {
  return OLAPcore_vwm_dv(dimvec_array, fk_array, orders, dimvec_nums, factor, size_lineorder,
                         group_nums, M1, M2, nthreads);
}

// OLAPcore_vwm_sv (:1258).
int ref_OLAPcore_vwm_sv(int8_t** dimvec_array, int32_t** fk_array, int* orders, int dimvec_nums,
                        int* factor, int size_lineorder, int group_nums, int32_t* M1, int32_t* M2,
                        int nthreads) {
  return OLAPcore_vwm_sv(dimvec_array, fk_array, orders, dimvec_nums, factor, size_lineorder,
                         group_nums, M1, M2, nthreads);
}

// join_cwm_sv (:908) + agg_cwm_sv (:764); groupID must hold size_lineorder entries.
int ref_OLAPcore_cwm_sv(int8_t** dimvec_array, int32_t** fk_array, int* orders, int dimvec_nums,
                        int* factor, int size_lineorder, int group_nums, int32_t* M1, int32_t* M2,
                        int16_t* groupID, int nthreads) {
  join_cwm_sv(dimvec_array, fk_array, orders, dimvec_nums, groupID, factor, size_lineorder, nthreads);
  return agg_cwm_sv(groupID, size_lineorder, M1, M2, group_nums, nthreads);
}

// join_cwm_dv (:840) + agg_cwm_dv (:685) with internally allocated per-thread lists.
int ref_OLAPcore_cwm_dv(int8_t** dimvec_array, int32_t** fk_array, int* orders, int dimvec_nums,
                        int* factor, int size_lineorder, int group_nums, int32_t* M1, int32_t* M2,
                        int nthreads) {
  std::vector<int64_t*> oid(nthreads);
  std::vector<int16_t*> gid(nthreads);
  std::vector<int> index(nthreads, 0);
  for (int i = 0; i < nthreads; i++) {
    oid[i] = new int64_t[size_lineorder];
    gid[i] = new int16_t[size_lineorder];
  }
  join_cwm_dv(dimvec_array, fk_array, orders, dimvec_nums, oid.data(), gid.data(), factor,
              index.data(), size_lineorder, nthreads);
  int r = agg_cwm_dv(oid.data(), gid.data(), index.data(), size_lineorder, M1, M2, group_nums,
                     nthreads);
  for (int i = 0; i < nthreads; i++) {
    delete[] oid[i];
    delete[] gid[i];
  }
  return r;
}

// Per-group sums of the reference's vector-wise static-vector thread body
// (:509-568) over [start, start + num_tuples), into a caller-zeroed uint32
// group_vector.  Requires group_nums <= 32766 (int16 group ids).
void ref_vwm_sv_groups(int8_t** dimvec_array, int32_t** fk_array, int* orders, int dimvec_nums,
                       int* factor, int64_t start, int64_t num_tuples, int32_t* M1, int32_t* M2,
                       uint32_t* group_vector) {
  std::vector<int16_t> gid(size_v);
  pth_vwmolapcoret a;
  std::memset(&a, 0, sizeof(a));
  a.start = start;
  a.num_tuples = num_tuples;
  a.dimvec_array = dimvec_array;
  a.fk_array = fk_array;
  a.dimvec_nums = dimvec_nums;
  a.orders = orders;
  a.groupID = gid.data();
  a.group_vector = group_vector;
  a.M1 = M1;
  a.M2 = M2;
  a.factor = factor;
  OLAPcore_vwm_sv_thread(&a);
}

// Per-group sums of the reference's row-wise thread body (:329-367) over
// [0, num_tuples): int group ids (any group count).  The body reads M1[i]
// with the thread-local index, which equals the row only from start 0.
void ref_row_groups(int8_t** dimvec_array, int32_t** fk_array, int* orders, int dimvec_nums,
                    int* factor, int64_t num_tuples, int32_t* M1, int32_t* M2,
                    uint32_t* group_vector) {
  pth_rowolapcoret a;
  std::memset(&a, 0, sizeof(a));
  a.start = 0;
  a.num_tuples = num_tuples;
  a.dimvec_array = dimvec_array;
  a.fk_array = fk_array;
  a.dimvec_nums = dimvec_nums;
  a.orders = orders;
  a.group_vector = group_vector;
  a.M1 = M1;
  a.M2 = M2;
  a.factor = factor;
  OLAPcore_row_thread(&a);
}

// The reference's data generator (include/gendata_util.hpp:449-542) from the
// C library's default seed, copied into caller buffers; dimvec[t] receives
// size+1 bytes, the last one 0.
int ref_gen_data_olapcore(double sf, const double* sele, const int* bitmap, const int* groups,
                          int8_t** dimvec_out, int32_t** fk_out, int32_t* m1_out, int32_t* m2_out) {
  int8_t *dc, *ds, *dp, *dd;
  int32_t *fc, *fs, *fp, *fd, *M1, *M2;
  srand(1);
  std::streambuf* old = std::cout.rdbuf(nullptr);
  gen_data(sele[0], sele[1], sele[2], sele[3], sf, bitmap[0], bitmap[1], bitmap[2], bitmap[3],
           groups[0], groups[1], groups[2], groups[3], dc, ds, dp, dd, fc, fs, fp, fd, M1, M2);
  std::cout.rdbuf(old);
  int8_t* dv[4] = {dc, ds, dp, dd};
  int32_t* fk[4] = {fc, fs, fp, fd};
  const int n = size_of_table(TABLE_NAME::lineorder, sf);
  for (int t = 0; t < 4; t++) {
    const int sz = size_of_table(static_cast<TABLE_NAME>(t), sf);
    std::memcpy(dimvec_out[t], dv[t], sz);
    dimvec_out[t][sz] = 0;
    std::memcpy(fk_out[t], fk[t], sizeof(int32_t) * n);
    delete[] dv[t];
    delete[] fk[t];
  }
  std::memcpy(m1_out, M1, sizeof(int32_t) * n);
  std::memcpy(m2_out, M2, sizeof(int32_t) * n);
  delete[] M1;
  delete[] M2;
  return 0;
}

}  // extern "C"
