// ref_shim.cpp — test infrastructure only (oracle side).
//
// extern "C" wrappers around the UNMODIFIED reference scalar library
// (RVVLASparse src/scalar/*.cpp, compiled from its own sources by
// oracle/Makefile into oracle/_ref/libref_scalar.so).  Nothing in the product
// path links this file: tests use it to pin the oracle restatement, the
// golden-fixture script uses it to write tests/golden/, and bench.py's CPU
// baseline times it.
//
// Every wrapper builds the reference's own container type (spMtxCRS,
// spMtxHCSR, spMtxSELL_C_Sigma, spMtxLAV, spMtxCVR — include/*.h of the
// reference) and calls the reference's explicit specialisation
//   sparse_mv<T, Fmt, false, stage>   (include/spmv_mtx.h:21-29)
//   convert<T, spMtxHCSR, false>      (src/scalar/crs_to_hcsr.cpp:137-169)
// so the arithmetic measured and compared is the reference's, not ours.
#include "sparse_matrix.h"

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <exception>
#include <string>
#include <vector>
#include <omp.h>

using namespace SparseMatrixLib;

// Built twice by oracle/Makefile: into libref_scalar.so with the defaults
// (the reference's scalar specialisations sparse_mv<T, Fmt, false>, names
// refx_*) and into libref_rvv.so with -DREFX_SIMD=true -DREFX_PREFIX=refr_
// (its RVV specialisations sparse_mv<T, Fmt, true> from src/rvv/, on the
// scalar intrinsic stand-in, names refr_*).  Builders stay the scalar ones.
#ifndef REFX_SIMD
#define REFX_SIMD false
#endif
#ifndef REFX_PREFIX
#define REFX_PREFIX refx_
#endif
#define REFX_CAT2(a, b) a##b
#define REFX_CAT(a, b) REFX_CAT2(a, b)
#define REFX_FN(name) REFX_CAT(REFX_PREFIX, name)

namespace {

thread_local std::string g_last_error;

template <class T>
struct CrsBox {
  spMtxCRS<T> A;
  std::vector<T> b, y;
};

template <class T>
CrsBox<T>* crs_new(int64_t m, int64_t n, int64_t nz, const int* Rst, const int* Col, const T* Val) {
  auto* box = new CrsBox<T>();
  // spMtxCRS(m, n, nz, Rst, Col, Val) copies the arrays (include/CRS.h:67-76).
  box->A = spMtxCRS<T>((size_t)m, (size_t)n, (size_t)nz, Rst, Col, Val);
  box->b.assign((size_t)n, T(0));
  box->y.assign((size_t)m, T(0));
  return box;
}

template <class M, class T>
struct FmtBox {
  M A;
  std::vector<T> b, y;
};

template <class Box, class Fn>
double time_loop(Box* box, int iters, Fn&& fn) {
  // Median of `iters` timed calls (steady_clock), after one warm-up call.
  fn();
  std::vector<double> t((size_t)iters);
  for (int i = 0; i < iters; ++i) {
    auto t0 = std::chrono::steady_clock::now();
    fn();
    auto t1 = std::chrono::steady_clock::now();
    t[(size_t)i] = std::chrono::duration<double>(t1 - t0).count();
  }
  std::sort(t.begin(), t.end());
  return t[(size_t)iters / 2];
}

}  // namespace

extern "C" {

const char* REFX_FN(last_error)() { return g_last_error.c_str(); }
int REFX_FN(num_threads)() { return omp_get_max_threads(); }

// ---------------------------------------------------------------- CRS
#define REFX_CRS(VT, S)                                                                       \
  void* REFX_FN(crs_new_##S)(int64_t m, int64_t n, int64_t nz, const int* Rst, const int* Col,   \
                         const VT* Val) {                                                     \
    return crs_new<VT>(m, n, nz, Rst, Col, Val);                                              \
  }                                                                                          \
  void REFX_FN(crs_free_##S)(void* h) { delete (CrsBox<VT>*)h; }                                  \
  int REFX_FN(crs_spmv_##S)(void* h, VT alpha, const VT* b, VT beta, VT* y) {                        \
    auto* box = (CrsBox<VT>*)h;                                                               \
    std::memcpy(box->b.data(), b, box->b.size() * sizeof(VT));                                \
    std::memcpy(box->y.data(), y, box->y.size() * sizeof(VT));                                \
    sparse_matrix_status st = sparse_mv<VT, spMtxCRS, REFX_SIMD>(                                 \
        SPARSE_OPERATION_NON_TRANSPOSE, alpha, box->A, sparse_matrix_descr{}, box->b, beta,  \
        box->y);                                                                             \
    std::memcpy(y, box->y.data(), box->y.size() * sizeof(VT));                                \
    return st.code;                                                                          \
  }                                                                                          \
  double REFX_FN(crs_time_##S)(void* h, VT alpha, const VT* b, VT beta, int iters) {                \
    auto* box = (CrsBox<VT>*)h;                                                               \
    std::memcpy(box->b.data(), b, box->b.size() * sizeof(VT));                                \
    return time_loop(box, iters, [&] {                                                       \
      sparse_mv<VT, spMtxCRS, REFX_SIMD>(SPARSE_OPERATION_NON_TRANSPOSE, alpha, box->A,           \
                                    sparse_matrix_descr{}, box->b, beta, box->y);            \
    });                                                                                      \
  }
REFX_CRS(double, f64)
REFX_CRS(float, f32)

// ---------------------------------------------------------------- HCSR
// info[0..6] = R, C, m, n, nz, b_m, b_n ; sizes[0..4] = |block_ptr|, |row_offset|,
// |row_ptr|, |col_idx|, |values|
#define REFX_HCSR(VT, S)                                                                      \
  void* REFX_FN(hcsr_convert_##S)(void* crs, int R, int C, double p, int set_R, int set_C,       \
                              int set_p) {                                                   \
    auto* src = (CrsBox<VT>*)crs;                                                             \
    auto* box = new FmtBox<spMtxHCSR<VT>, VT>();                                               \
    convertParams params;                                                                    \
    if (set_R) { convertValue v; v.i = R; params.param["R"] = v; }                           \
    if (set_C) { convertValue v; v.i = C; params.param["C"] = v; }                           \
    if (set_p) { convertValue v; v.d = p; params.param["p"] = v; }                           \
    try {                                                                                    \
      convert<VT, spMtxHCSR, false>(box->A, src->A, params);                                  \
    } catch (const std::exception& e) {                                                      \
      g_last_error = e.what();                                                               \
      delete box;                                                                            \
      return nullptr;                                                                        \
    }                                                                                        \
    box->b.assign(box->A.n, VT(0));                                                           \
    box->y.assign(box->A.m, VT(0));                                                           \
    return box;                                                                              \
  }                                                                                          \
  void* REFX_FN(hcsr_new_##S)(const int64_t* info, const int* block_ptr,                         \
                          const uint32_t* row_offset, const uint32_t* row_ptr,               \
                          const uint16_t* col_idx, const VT* values, const int64_t* sizes) {  \
    auto* box = new FmtBox<spMtxHCSR<VT>, VT>();                                               \
    auto& A = box->A;                                                                        \
    A.R = (size_t)info[0]; A.C = (size_t)info[1]; A.m = (size_t)info[2];                     \
    A.n = (size_t)info[3]; A.nz = (size_t)info[4]; A.b_m = (size_t)info[5];                  \
    A.b_n = (size_t)info[6];                                                                 \
    A.block_ptr.assign(block_ptr, block_ptr + sizes[0]);                                     \
    A.row_offset.assign(row_offset, row_offset + sizes[1]);                                  \
    A.row_ptr.assign(row_ptr, row_ptr + sizes[2]);                                           \
    A.col_idx.assign(col_idx, col_idx + sizes[3]);                                           \
    A.values.assign(values, values + sizes[4]);                                              \
    box->b.assign(A.n, VT(0));                                                                \
    box->y.assign(A.m, VT(0));                                                                \
    return box;                                                                              \
  }                                                                                          \
  void REFX_FN(hcsr_free_##S)(void* h) { delete (FmtBox<spMtxHCSR<VT>, VT>*)h; }                   \
  void REFX_FN(hcsr_info_##S)(void* h, int64_t* info, int64_t* sizes) {                          \
    auto& A = ((FmtBox<spMtxHCSR<VT>, VT>*)h)->A;                                              \
    info[0] = (int64_t)A.R; info[1] = (int64_t)A.C; info[2] = (int64_t)A.m;                  \
    info[3] = (int64_t)A.n; info[4] = (int64_t)A.nz; info[5] = (int64_t)A.b_m;               \
    info[6] = (int64_t)A.b_n;                                                                \
    sizes[0] = (int64_t)A.block_ptr.size(); sizes[1] = (int64_t)A.row_offset.size();         \
    sizes[2] = (int64_t)A.row_ptr.size(); sizes[3] = (int64_t)A.col_idx.size();              \
    sizes[4] = (int64_t)A.values.size();                                                     \
  }                                                                                          \
  void REFX_FN(hcsr_export_##S)(void* h, int* block_ptr, uint32_t* row_offset,                   \
                            uint32_t* row_ptr, uint16_t* col_idx, VT* values) {               \
    auto& A = ((FmtBox<spMtxHCSR<VT>, VT>*)h)->A;                                              \
    std::memcpy(block_ptr, A.block_ptr.data(), A.block_ptr.size() * sizeof(int));            \
    std::memcpy(row_offset, A.row_offset.data(), A.row_offset.size() * sizeof(uint32_t));    \
    std::memcpy(row_ptr, A.row_ptr.data(), A.row_ptr.size() * sizeof(uint32_t));             \
    std::memcpy(col_idx, A.col_idx.data(), A.col_idx.size() * sizeof(uint16_t));             \
    std::memcpy(values, A.values.data(), A.values.size() * sizeof(VT));                       \
  }                                                                                          \
  int REFX_FN(hcsr_spmv_##S)(void* h, VT alpha, const VT* b, VT beta, VT* y) {                       \
    auto* box = (FmtBox<spMtxHCSR<VT>, VT>*)h;                                                 \
    std::memcpy(box->b.data(), b, box->b.size() * sizeof(VT));                                \
    std::memcpy(box->y.data(), y, box->y.size() * sizeof(VT));                                \
    sparse_matrix_status st = sparse_mv<VT, spMtxHCSR, REFX_SIMD>(                                \
        SPARSE_OPERATION_NON_TRANSPOSE, alpha, box->A, sparse_matrix_descr{}, box->b, beta,  \
        box->y);                                                                             \
    std::memcpy(y, box->y.data(), box->y.size() * sizeof(VT));                                \
    return st.code;                                                                          \
  }                                                                                          \
  double REFX_FN(hcsr_time_##S)(void* h, VT alpha, const VT* b, VT beta, int iters) {               \
    auto* box = (FmtBox<spMtxHCSR<VT>, VT>*)h;                                                 \
    std::memcpy(box->b.data(), b, box->b.size() * sizeof(VT));                                \
    return time_loop(box, iters, [&] {                                                       \
      sparse_mv<VT, spMtxHCSR, REFX_SIMD>(SPARSE_OPERATION_NON_TRANSPOSE, alpha, box->A,          \
                                     sparse_matrix_descr{}, box->b, beta, box->y);           \
    });                                                                                      \
  }
REFX_HCSR(double, f64)
REFX_HCSR(float, f32)

// ---------------------------------------------------------------- SELL-C-sigma
// ints[0..5] = m, n, cnt_b, nz, C, Sigma ; len = |vCol| = |vVal|
#define REFX_SELL(VT, S)                                                                      \
  void* REFX_FN(sell_new_##S)(const int64_t* ints, const int* vCl, const int* vCs, const int* vBs, \
                          const int* vSBs, const uint32_t* vCol, const uint32_t* vPerm,      \
                          const VT* vVal, int64_t len) {                                      \
    auto* box = new FmtBox<spMtxSELL_C_Sigma<VT>, VT>();                                       \
    auto& A = box->A;                                                                        \
    A.m = (size_t)ints[0]; A.n = (size_t)ints[1]; A.cnt_b = (size_t)ints[2];                 \
    A.nz = (size_t)ints[3]; A.C = (int)ints[4]; A.Sigma = (int)ints[5];                      \
    A.vCl.assign(vCl, vCl + A.cnt_b); A.vCs.assign(vCs, vCs + A.cnt_b);                      \
    A.vBs.assign(vBs, vBs + A.cnt_b); A.vSBs.assign(vSBs, vSBs + A.cnt_b);                   \
    A.vCol.assign(vCol, vCol + len); A.vVal.assign(vVal, vVal + len);                        \
    A.vPerm.assign(vPerm, vPerm + A.m);                                                      \
    box->b.assign(A.n, VT(0));                                                                \
    box->y.assign(A.m, VT(0));                                                                \
    return box;                                                                              \
  }                                                                                          \
  void REFX_FN(sell_free_##S)(void* h) { delete (FmtBox<spMtxSELL_C_Sigma<VT>, VT>*)h; }           \
  int REFX_FN(sell_spmv_##S)(void* h, int stage, VT alpha, const VT* b, VT beta, VT* y) {            \
    auto* box = (FmtBox<spMtxSELL_C_Sigma<VT>, VT>*)h;                                         \
    std::memcpy(box->b.data(), b, box->b.size() * sizeof(VT));                                \
    std::memcpy(box->y.data(), y, box->y.size() * sizeof(VT));                                \
    sparse_matrix_status st;                                                                 \
    auto op = SPARSE_OPERATION_NON_TRANSPOSE;                                                \
    auto d = sparse_matrix_descr{};                                                          \
    switch (stage) {                                                                         \
      case 0: st = sparse_mv<VT, spMtxSELL_C_Sigma, REFX_SIMD, SPARSE_MATRIX_MV_PREPARATION>(     \
                  op, alpha, box->A, d, box->b, beta, box->y); break;                        \
      case 1: st = sparse_mv<VT, spMtxSELL_C_Sigma, REFX_SIMD, SPARSE_MATRIX_MV_MULT>(            \
                  op, alpha, box->A, d, box->b, beta, box->y); break;                        \
      case 2: st = sparse_mv<VT, spMtxSELL_C_Sigma, REFX_SIMD, SPARSE_MATRIX_MV_GET_RESULTS>(     \
                  op, alpha, box->A, d, box->b, beta, box->y); break;                        \
      default: st = sparse_mv<VT, spMtxSELL_C_Sigma, REFX_SIMD, SPARSE_MATRIX_MV_ALL_STAGES>(     \
                  op, alpha, box->A, d, box->b, beta, box->y); break;                        \
    }                                                                                        \
    std::memcpy(y, box->y.data(), box->y.size() * sizeof(VT));                                \
    return st.code;                                                                          \
  }                                                                                          \
  double REFX_FN(sell_time_##S)(void* h, VT alpha, const VT* b, VT beta, int iters) {               \
    auto* box = (FmtBox<spMtxSELL_C_Sigma<VT>, VT>*)h;                                         \
    std::memcpy(box->b.data(), b, box->b.size() * sizeof(VT));                                \
    return time_loop(box, iters, [&] {                                                       \
      sparse_mv<VT, spMtxSELL_C_Sigma, REFX_SIMD, SPARSE_MATRIX_MV_ALL_STAGES>(                   \
          SPARSE_OPERATION_NON_TRANSPOSE, alpha, box->A, sparse_matrix_descr{}, box->b,      \
          beta, box->y);                                                                     \
    });                                                                                      \
  }
REFX_SELL(double, f64)
REFX_SELL(float, f32)

// ---------------------------------------------------------------- LAV
// ints[0..7] = SIMD_Lanes, m, n, nz, segment_count, chunk_count, segment_len, (unused)
// lens[0..6] = |chunk_offsets|, |chunk_offsets_full_mask|, |segment_ptr|, |out_order|,
//              |mask|, |val| (= |col_id|), sparse nz
#define REFX_LAV(VT, S)                                                                       \
  void* REFX_FN(lav_new_##S)(const int64_t* ints, double Tthr, const int64_t* lens,              \
                         const int* chunk_offsets, const int* chunk_offsets_full_mask,       \
                         const uint64_t* segment_ptr, const uint32_t* out_order,             \
                         const uint16_t* mask, const VT* val, const uint32_t* col_id,         \
                         const int* sp_Rst, const int* sp_Col, const VT* sp_Val) {            \
    auto* box = new FmtBox<spMtxLAV<VT>, VT>();                                                \
    auto& A = box->A;                                                                        \
    A.SIMD_Lanes = (size_t)ints[0]; A.m = (int)ints[1]; A.n = (int)ints[2];                  \
    A.nz = (int)ints[3]; A.segment_count = (size_t)ints[4]; A.chunk_count = (size_t)ints[5]; \
    A.segment_len = (int)ints[6]; A.T = Tthr;                                                \
    A.chunk_offsets.assign(chunk_offsets, chunk_offsets + lens[0]);                          \
    A.chunk_offsets_full_mask.assign(chunk_offsets_full_mask,                                \
                                     chunk_offsets_full_mask + lens[1]);                     \
    A.segment_ptr.assign(segment_ptr, segment_ptr + lens[2]);                                \
    A.out_order.assign(out_order, out_order + lens[3]);                                      \
    A.mask.assign(mask, mask + lens[4]);                                                     \
    A.val.assign(val, val + lens[5]);                                                        \
    A.col_id.assign(col_id, col_id + lens[5]);                                               \
    A.sparse_part = spMtxCRS<VT>((size_t)A.m, (size_t)A.n, (size_t)lens[6], sp_Rst, sp_Col,   \
                                sp_Val);                                                     \
    box->b.assign((size_t)A.n, VT(0));                                                        \
    box->y.assign((size_t)A.m, VT(0));                                                        \
    return box;                                                                              \
  }                                                                                          \
  void REFX_FN(lav_free_##S)(void* h) { delete (FmtBox<spMtxLAV<VT>, VT>*)h; }                     \
  int REFX_FN(lav_spmv_##S)(void* h, VT alpha, const VT* b, VT beta, VT* y) {                        \
    auto* box = (FmtBox<spMtxLAV<VT>, VT>*)h;                                                  \
    std::memcpy(box->b.data(), b, box->b.size() * sizeof(VT));                                \
    std::memcpy(box->y.data(), y, box->y.size() * sizeof(VT));                                \
    sparse_matrix_status st = sparse_mv<VT, spMtxLAV, REFX_SIMD>(                                 \
        SPARSE_OPERATION_NON_TRANSPOSE, alpha, box->A, sparse_matrix_descr{}, box->b, beta,  \
        box->y);                                                                             \
    std::memcpy(y, box->y.data(), box->y.size() * sizeof(VT));                                \
    return st.code;                                                                          \
  }                                                                                          \
  double REFX_FN(lav_time_##S)(void* h, VT alpha, const VT* b, VT beta, int iters) {                \
    auto* box = (FmtBox<spMtxLAV<VT>, VT>*)h;                                                  \
    std::memcpy(box->b.data(), b, box->b.size() * sizeof(VT));                                \
    return time_loop(box, iters, [&] {                                                       \
      sparse_mv<VT, spMtxLAV, REFX_SIMD>(SPARSE_OPERATION_NON_TRANSPOSE, alpha, box->A,           \
                                    sparse_matrix_descr{}, box->b, beta, box->y);            \
    });                                                                                      \
  }
REFX_LAV(double, f64)
REFX_LAV(float, f32)

// src/rvv/spmv_mtx_cvr.cpp of the reference holds the scalar product again
// (sparse_mv<T, spMtxCVR, false> only, :22 and :72): there is no simd = true
// CVR, so the RVV build of this shim (-DREFX_SKIP_CVR=1) leaves CVR out.
#if !defined(REFX_SKIP_CVR) || !REFX_SKIP_CVR
// ---------------------------------------------------------------- CVR
// ints[0..5] = nItems, numRows, numCols, SIMD_LEN, Nthreads, Nthreads_avail
// lens[0..2] = |vPack_vec_vals| (= |cols|), |vPack_vec_record|, |writeback_pos_record|
#define REFX_CVR(VT, S)                                                                       \
  void* REFX_FN(cvr_new_##S)(const int64_t* ints, const int64_t* lens, const VT* vals,            \
                         const uint32_t* cols, const int* record, const int* writeback) {    \
    auto* box = new FmtBox<spMtxCVR<VT>, VT>();                                                \
    auto& A = box->A;                                                                        \
    A.nItems = (size_t)ints[0]; A.numRows = (size_t)ints[1]; A.numCols = (size_t)ints[2];    \
    A.SIMD_LEN = (size_t)ints[3]; A.Nthreads = (int)ints[4]; A.Nthreads_avail = (int)ints[5];\
    A.vPack_vec_vals.assign(vals, vals + lens[0]);                                           \
    A.vPack_vec_cols.assign(cols, cols + lens[0]);                                           \
    A.vPack_vec_record.assign(record, record + lens[1]);                                     \
    A.writeback_pos_record.assign(writeback, writeback + lens[2]);                           \
    box->b.assign(A.numCols, VT(0));                                                          \
    box->y.assign(A.numRows, VT(0));                                                          \
    return box;                                                                              \
  }                                                                                          \
  void REFX_FN(cvr_free_##S)(void* h) { delete (FmtBox<spMtxCVR<VT>, VT>*)h; }                     \
  int REFX_FN(cvr_spmv_##S)(void* h, VT alpha, const VT* b, VT beta, VT* y) {                        \
    auto* box = (FmtBox<spMtxCVR<VT>, VT>*)h;                                                  \
    std::memcpy(box->b.data(), b, box->b.size() * sizeof(VT));                                \
    std::memcpy(box->y.data(), y, box->y.size() * sizeof(VT));                                \
    sparse_matrix_status st = sparse_mv<VT, spMtxCVR, REFX_SIMD>(                                 \
        SPARSE_OPERATION_NON_TRANSPOSE, alpha, box->A, sparse_matrix_descr{}, box->b, beta,  \
        box->y);                                                                             \
    std::memcpy(y, box->y.data(), box->y.size() * sizeof(VT));                                \
    return st.code;                                                                          \
  }                                                                                          \
  double REFX_FN(cvr_time_##S)(void* h, VT alpha, const VT* b, VT beta, int iters) {                \
    auto* box = (FmtBox<spMtxCVR<VT>, VT>*)h;                                                  \
    std::memcpy(box->b.data(), b, box->b.size() * sizeof(VT));                                \
    return time_loop(box, iters, [&] {                                                       \
      sparse_mv<VT, spMtxCVR, REFX_SIMD>(SPARSE_OPERATION_NON_TRANSPOSE, alpha, box->A,           \
                                    sparse_matrix_descr{}, box->b, beta, box->y);            \
    });                                                                                      \
  }
REFX_CVR(double, f64)
REFX_CVR(float, f32)
#endif

}  // extern "C"
