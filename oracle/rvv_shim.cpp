// rvv_shim.cpp — test infrastructure only (oracle side).
//
// extern "C" wrappers around the reference's UNMODIFIED RVV-only kernels
// (RVVLASparse src/rvv/spmv_mtx_csr5.cpp, src/rvv/spmv_mtx_vnec.cpp,
// src/rvv/spmv_vhcc.cpp), compiled from their own sources for x86-64 by
// oracle/Makefile target `ref-rvv` against the scalar intrinsic stand-in
// oracle/rvv_emul/riscv_vector.h (VLEN 256) into oracle/_ref/libref_rvv.so.
// Tests use them to pin the oracle's restatements of these three kernels to
// the reference's own code; nothing in the product path links this file.
//
// CSR5 and VHCC have no builder in the reference (asCSR5 is declared in
// include/CSR5.h:61-65 and never defined; VHCC has only setters,
// include/VHCC.h:80-112), so their objects are filled from layouts the
// oracle's builders produced.  VNEC is built by the reference's own
// constructor spMtxVNEC(const spMtxCRS&) (include/VNEC.h:200-227), which
// also picks the variant (D, S or L).  Every call goes through the
// reference's explicit specialisation sparse_mv<T, Fmt, true, stage>.
#include "riscv_vector.h"
#include "sparse_matrix.h"

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <exception>
#include <string>
#include <vector>
#include <omp.h>

using namespace SparseMatrixLib;

namespace {

thread_local std::string g_last_error;

template <class M, class T>
struct Box {
  M A;
  std::vector<T> b, y;
};

template <class T>
struct VnecBox {
  spMtxCRS<T> G;
  spMtxVNEC<T>* A = nullptr;
  std::vector<T> b, y;
  ~VnecBox() { delete A; }
};

template <class T, class M, class Fn>
int run(M& box, T alpha, const T* b, T beta, T* y, Fn&& call) {
  try {
    std::memcpy(box.b.data(), b, box.b.size() * sizeof(T));
    std::memcpy(box.y.data(), y, box.y.size() * sizeof(T));
    const sparse_matrix_status st = call(alpha, beta);
    std::memcpy(y, box.y.data(), box.y.size() * sizeof(T));
    return st.code;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return -1;
  }
}

}  // namespace

extern "C" {

const char* refv_last_error() { return g_last_error.c_str(); }
int refv_num_threads() { return omp_get_max_threads(); }
int refv_vlen() { return RVV_EMUL_VLEN; }

// ---------------------------------------------------------------- CSR5
// ints[0..10] = m, n, nnz, bit_y_offset, bit_seg_offset, tile_desc_len,
//               tail_tile_start, p, omega, sigma, num_offsets
// lens[0..5]  = |csr_row_pointer|, |csr_column_index| (= |csr_value|),
//               |tile_pointer|, |tile_descriptor|, |tile_empty_offset_pointer|,
//               |tile_empty_offset|
#define REFV_CSR5(VT, S)                                                                      \
  void* refv_csr5_new_##S(const int64_t* ints, const int64_t* lens, const int* row_ptr,       \
                          const uint32_t* col, const VT* val, const uint32_t* tile_ptr,       \
                          const uint32_t* tile_desc, const uint32_t* teo_ptr,                 \
                          const uint32_t* teo) {                                              \
    auto* box = new Box<spMtxCSR5<VT>, VT>();                                                 \
    auto& A = box->A;                                                                         \
    A._m = (int)ints[0]; A._n = (int)ints[1]; A._nnz = (int)ints[2];                          \
    A._bit_y_offset = (int)ints[3]; A._bit_seg_offset = (int)ints[4];                         \
    A._tile_desc_len = (int)ints[5]; A._tail_tile_start = (int)ints[6]; A._p = (int)ints[7];  \
    A._omega = (int)ints[8]; A._sigma = (int)ints[9]; A._num_offsets = (int)ints[10];         \
    A._csr_row_pointer.assign(row_ptr, row_ptr + lens[0]);                                    \
    A._csr_column_index.assign(col, col + lens[1]);                                           \
    A._csr_value.assign(val, val + lens[1]);                                                  \
    A._csr5_tile_pointer.assign(tile_ptr, tile_ptr + lens[2]);                                \
    A._csr5_tile_descriptor.assign(tile_desc, tile_desc + lens[3]);                           \
    A._csr5_tile_empty_offset_pointer.assign(teo_ptr, teo_ptr + lens[4]);                     \
    A._csr5_tile_empty_offset.assign(teo, teo + lens[5]);                                     \
    /* one cache line per OpenMP thread (the kernel clears and indexes it that way) */        \
    A._temp_calibrator.assign((size_t)omp_get_max_threads() * CSR5_CACHELINE / sizeof(VT),    \
                              VT(0));                                                         \
    box->b.assign((size_t)A._n, VT(0));                                                       \
    box->y.assign((size_t)A._m, VT(0));                                                       \
    return box;                                                                               \
  }                                                                                           \
  void refv_csr5_free_##S(void* h) { delete (Box<spMtxCSR5<VT>, VT>*)h; }                     \
  /* threads > 0: the default OpenMP team size for the call (the kernel sizes its */         \
  /* tile split and calibrator by omp_get_max_threads()).                          */         \
  int refv_csr5_spmv_##S(void* h, int threads, VT alpha, const VT* b, VT beta, VT* y) {       \
    auto& box = *(Box<spMtxCSR5<VT>, VT>*)h;                                                  \
    const int saved = omp_get_max_threads();                                                  \
    if (threads > 0) omp_set_num_threads(threads);                                            \
    if ((size_t)omp_get_max_threads() * CSR5_CACHELINE / sizeof(VT) >                         \
        box.A._temp_calibrator.size())                                                        \
      box.A._temp_calibrator.assign((size_t)omp_get_max_threads() * CSR5_CACHELINE /          \
                                    sizeof(VT), VT(0));                                       \
    const int rc = run(box, alpha, b, beta, y, [&](VT a, VT be) {                             \
      return sparse_mv<VT, spMtxCSR5, true>(SPARSE_OPERATION_NON_TRANSPOSE, a, box.A,         \
                                            sparse_matrix_descr{}, box.b, be, box.y);         \
    });                                                                                       \
    omp_set_num_threads(saved);                                                               \
    return rc;                                                                                \
  }
REFV_CSR5(double, f64)
REFV_CSR5(float, f32)

// ---------------------------------------------------------------- VHCC
// ints[0..7] = num_rows, num_cols, num_entries, num_vectors, pad_entries,
//              pad_rows, num_threads, vec_size
// lens[0..4] = |thr_info| (ints, 10 per thread), |veceor_ptr|,
//              |scan_mask| (bytes), |row_arr|, |col_arr| (= |vals_arr|)
#define REFV_VHCC(VT, S)                                                                      \
  void* refv_vhcc_new_##S(const int64_t* ints, const int64_t* lens, const int32_t* thr,       \
                          const uint32_t* veceor, const uint8_t* scan_mask,                   \
                          const uint32_t* row_arr, const uint32_t* col_arr, const VT* vals) { \
    auto* box = new Box<spMtxVHCC<VT>, VT>();                                                 \
    auto& A = box->A;                                                                         \
    A.set_params(vhcc_params((size_t)ints[6], 1, 512, 512, (size_t)ints[7]));                 \
    A.set_properties((size_t)ints[0], (size_t)ints[1], (size_t)ints[2], (size_t)ints[3],      \
                     (size_t)ints[4], (size_t)ints[5]);                                       \
    auto& ti = A.get_thr_info_reference();                                                    \
    ti.resize((size_t)lens[0] / 10);                                                          \
    static_assert(sizeof(thr_info_t) == 10 * sizeof(int32_t), "thr_info_t layout");           \
    if (!ti.empty()) std::memcpy(ti.data(), thr, ti.size() * sizeof(thr_info_t));             \
    A.get_veceor_reference().assign(veceor, veceor + lens[1]);                                \
    A.get_scan_mask_reference().assign(scan_mask, scan_mask + lens[2]);                       \
    A.get_row_arr_reference().assign(row_arr, row_arr + lens[3]);                             \
    A.get_col_arr_reference().assign(col_arr, col_arr + lens[4]);                             \
    A.get_vals_arr_reference().assign(vals, vals + lens[4]);                                  \
    box->b.assign((size_t)ints[1], VT(0));                                                    \
    box->y.assign((size_t)ints[0], VT(0));                                                    \
    return box;                                                                               \
  }                                                                                           \
  void refv_vhcc_free_##S(void* h) { delete (Box<spMtxVHCC<VT>, VT>*)h; }                     \
  /* The fp64 alpha = 1, beta = 0 branch copies tmp_y to y in a parallel region */          \
  /* of the default team size (src/rvv/spmv_vhcc.cpp:385) while it splits y by    */          \
  /* vhcc_params.num_threads, so a larger default team writes past y: the default */          \
  /* team size is set to the structure's thread count around the call, the setting */         \
  /* the reference is run with (OMP_NUM_THREADS = num_threads).                    */         \
  int refv_vhcc_spmv_##S(void* h, VT alpha, const VT* b, VT beta, VT* y) {                    \
    auto& box = *(Box<spMtxVHCC<VT>, VT>*)h;                                                  \
    const int saved = omp_get_max_threads();                                                  \
    omp_set_num_threads((int)box.A.get_params().num_threads);                                 \
    const int rc = run(box, alpha, b, beta, y, [&](VT a, VT be) {                             \
      return sparse_mv<VT, spMtxVHCC, true>(SPARSE_OPERATION_NON_TRANSPOSE, a, box.A,         \
                                            sparse_matrix_descr{}, box.b, be, box.y);         \
    });                                                                                       \
    omp_set_num_threads(saved);                                                               \
    return rc;                                                                                \
  }
REFV_VHCC(double, f64)
REFV_VHCC(float, f32)

// ---------------------------------------------------------------- VNEC
// info[0..1] = vnec_t (0 D, 1 S, 2 L), NUM_THREADS_VNEC; *ird = IRD_mat
#define REFV_VNEC(VT, S)                                                                      \
  /* threads > 0: the OpenMP team size while the constructor runs (it sets    */           \
  /* NUM_THREADS_VNEC from it and computes IRD with that many threads).       */           \
  void* refv_vnec_new_##S(int64_t m, int64_t n, int64_t nz, const int* Rst, const int* Col,   \
                          const VT* Val, int threads) {                                       \
    try {                                                                                     \
      auto* box = new VnecBox<VT>();                                                          \
      box->G = spMtxCRS<VT>((size_t)m, (size_t)n, (size_t)nz, Rst, Col, Val);                 \
      const int saved = omp_get_max_threads();                                                \
      if (threads > 0) omp_set_num_threads(threads);                                          \
      box->A = new spMtxVNEC<VT>(box->G);                                                     \
      omp_set_num_threads(saved);                                                             \
      box->b.assign((size_t)n, VT(0));                                                        \
      box->y.assign((size_t)m, VT(0));                                                        \
      return box;                                                                             \
    } catch (const std::exception& e) {                                                       \
      g_last_error = e.what();                                                                \
      return nullptr;                                                                         \
    }                                                                                         \
  }                                                                                           \
  void refv_vnec_free_##S(void* h) { delete (VnecBox<VT>*)h; }                                \
  void refv_vnec_info_##S(void* h, int64_t* info, double* ird) {                              \
    auto& box = *(VnecBox<VT>*)h;                                                             \
    info[0] = (int64_t)box.A->vnec_t;                                                         \
    info[1] = (int64_t)box.A->NUM_THREADS_VNEC;                                               \
    *ird = (double)box.A->IRD_mat;                                                            \
  }                                                                                           \
  int refv_vnec_spmv_##S(void* h, VT alpha, const VT* b, VT beta, VT* y) {                    \
    auto& box = *(VnecBox<VT>*)h;                                                             \
    return run(box, alpha, b, beta, y, [&](VT a, VT be) {                                     \
      return sparse_mv<VT, spMtxVNEC, true>(SPARSE_OPERATION_NON_TRANSPOSE, a, *box.A,        \
                                            sparse_matrix_descr{}, box.b, be, box.y);         \
    });                                                                                       \
  }
REFV_VNEC(double, f64)
REFV_VNEC(float, f32)

// The reference's VNEC kernels read structures that no reference code fills
// (the constructor computes only IRD and the variant): this sets them from a
// layout the oracle's VNEC builder made for the same matrix, allocated the way
// the reference's freeMem() releases them (include/VNEC.h:265-319: malloc'd
// arrays, NUM_THREADS_VNEC + 1 slots for use_x_indices / ecr_xx_val, one
// malloc'd row list per thread in tasks), then selects the variant.
// ints[0..1] = vnec_t (0 D, 1 S, 2 L), NUM_THREADS_VNEC (<= 256, the D and L
//              kernels' carry arrays)
// lens[0..7] = |ecr_indices|, |use_x_indices|, |v_row_ptr|, |col_start|,
//              |val_align|, |tasks|, |row_begin| (= |row_end|), |reorder_col|
// Arrays a variant does not use may be NULL (their lengths 0).
}  // extern "C"
namespace {
template <class T>
T* dup(const T* src, int64_t n, int64_t pad = 0) {
  T* p = (T*)std::calloc((size_t)(n + pad > 0 ? n + pad : 1), sizeof(T));
  if (p && src && n > 0) std::memcpy(p, src, (size_t)n * sizeof(T));
  return p;
}
}  // namespace
extern "C" {
#define REFV_VNEC_FILL(VT, S)                                                                 \
  int refv_vnec_fill_##S(void* h, const int64_t* ints, const int64_t* lens, const int* tcs,    \
                         const int* tce, const int* nec, const int* ux_ptr, const int* ux,     \
                         const int* ecr, const int* vrp, const int* cs, const VT* va,          \
                         const int* tasks, const int* ts, const int* te, const int* sv,        \
                         const int* rb, const int* re, const int* rc, const VT* rv) {          \
    auto& A = *((VnecBox<VT>*)h)->A;                                                          \
    const int NT = (int)ints[1];                                                              \
    if (NT < 1 || NT > 256 || ints[0] < 0 || ints[0] > 2) {                                   \
      g_last_error = "refv_vnec_fill: bad variant or thread count";                            \
      return -1;                                                                              \
    }                                                                                         \
    A.freeMem();                                                                              \
    A.NUM_THREADS_VNEC = NT;                                                                  \
    A.vnec_t = (SpB_VNEC_type)ints[0];                                                        \
    A.thread_coord_start = (coord*)dup(tcs, 2 * (int64_t)NT);                                 \
    A.thread_coord_end = (coord*)dup(tce, 2 * (int64_t)NT);                                   \
    const int64_t nl = std::is_same<VT, float>::value ? nLanes_f32 : nLanes_f64;              \
    if (nec) {                                                                                \
      A.NEC_NUM = dup(nec, NT);                                                               \
      A.use_x_indices = (int**)std::calloc((size_t)NT + 1, sizeof(int*));                     \
      A.ecr_xx_val = (VT**)std::calloc((size_t)NT + 1, sizeof(VT*));                          \
      for (int t = 0; t < NT; ++t) {                                                          \
        A.use_x_indices[t] = dup(ux + ux_ptr[t], (int64_t)nec[t], nl);                        \
        A.ecr_xx_val[t] = dup<VT>(nullptr, (int64_t)nec[t], nl);                              \
      }                                                                                       \
    }                                                                                         \
    if (ecr) A.ecr_indices = dup(ecr, lens[0]);                                               \
    if (vrp) A.v_row_ptr = dup(vrp, lens[2]);                                                 \
    if (cs) A.col_start = dup(cs, lens[3]);                                                   \
    if (va) A.val_align = dup(va, lens[4]);                                                   \
    if (tasks) {                                                                              \
      A.tasks = (int**)std::calloc((size_t)NT, sizeof(int*));                                 \
      for (int t = 0; t < NT; ++t) {                                                          \
        const int64_t cnt = std::max<int64_t>((int64_t)te[t] - ts[t], (int64_t)sv[t]);        \
        const int64_t avail = std::max<int64_t>(0, std::min<int64_t>(cnt, lens[5] - ts[t]));  \
        A.tasks[t] = dup(tasks + ts[t], avail, cnt - avail + nl);                             \
      }                                                                                       \
      A.spvv_len = dup(sv, NT);                                                               \
      A.reorder_mat.task_start = dup(ts, NT);                                                 \
      A.reorder_mat.task_end = dup(te, NT);                                                   \
      A.reorder_mat.row_begin = dup(rb, lens[6], nl);                                         \
      A.reorder_mat.row_end = dup(re, lens[6], nl);                                           \
      A.reorder_mat.col = dup(rc, lens[7], nl);                                               \
      A.reorder_mat.nnz = dup(rv, lens[7], nl);                                               \
    }                                                                                         \
    return 0;                                                                                 \
  }
REFV_VNEC_FILL(double, f64)
REFV_VNEC_FILL(float, f32)

}  // extern "C"
