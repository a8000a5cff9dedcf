// vnec_build.h — host-side VNEC structure (see vnec_build.cpp).
#pragma once
#include <cstdint>
#include <vector>

namespace rvvla {

template <class T>
struct VnecHost {
  int NT = 0, nL = 0, variant = 0, max_nec = 0;
  float ird = 0.f;
  std::vector<int> tcs, tce;            // thread_coord_start / _end (x, y pairs)
  std::vector<int> ecr, nec, uxp, ux;   // compaction (D: merge pieces; S: row pieces)
  std::vector<int> vrp, cs;             // D: v_row_ptr, col_start
  std::vector<T> va;                    // D: val_align
  std::vector<int> tasks, ts, te, spv;  // S: tasks, task_start, task_end, spvv_len
  std::vector<int> rb, re, rc;          // S: reorder_mat row_begin/row_end/col
  std::vector<T> rv;                    // S: reorder_mat nnz
};

template <class T>
void vnec_build_host(const int* Rst, const int* Col, const T* Val, int64_t m, int64_t n, int64_t nnz, int64_t NT,
                     int force, int nL, double thr, VnecHost<T>& out);

}  // namespace rvvla
