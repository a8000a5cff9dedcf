// spmv_mtx.h — sparse_mv<T, Mtx, simd, stage> of the RVVLASparse API
// (include/spmv_mtx.h:19-29 of the reference): y = alpha*A*b + beta*y on the
// GPU for every format and every simd/stage combination.  Stages follow the
// reference: for SELL-C-sigma PREPARATION permutes y, MULT multiplies in the
// sorted row order, GET_RESULTS restores the order; for the other formats
// PREPARATION and GET_RESULTS do nothing and MULT is the whole product.
// beta == 0 does not read y.  The status code is 0 or an rvvla_status.
#pragma once
#include <stdexcept>
#include <vector>

#include "types.h"

namespace SparseMatrixLib {

template <class T, template <class> class Mtx, bool simd = true,
          sparse_matrix_mv_stage stage = SPARSE_MATRIX_MV_ALL_STAGES>
sparse_matrix_status sparse_mv(sparse_operation_t type_op, T alpha, const Mtx<T>& mat, sparse_matrix_descr descr,
                               const std::vector<T>& b, T beta, std::vector<T>& y) {
  (void)descr;
  return rvvla_sparse_mv(type_op, alpha, mat, b, beta, y, stage);  // argument-dependent lookup
}

// Mixed precision (an addition; the reference has no counterpart): the
// product of a float matrix (fp32 values) with fp32 b and y whose row sums run
// in compensated fp32 (two-sum) and whose partial sums of different tiles or
// blocks merge in fp64 — normwise error ~1e-8 against an fp64 product of the
// same values, where the plain fp32 product gives ~1e-6.  For spMtxCRS,
// spMtxHCSR, spMtxCSR5 and spMtxSELL_C_Sigma (all stages at once); op must
// be SPARSE_OPERATION_NON_TRANSPOSE.
template <template <class> class Mtx>
sparse_matrix_status sparse_mv_mixed(sparse_operation_t type_op, float alpha, const Mtx<float>& mat,
                                     sparse_matrix_descr descr, const std::vector<float>& b, float beta,
                                     std::vector<float>& y) {
  (void)descr;
  return rvvla_sparse_mv_mixed(type_op, alpha, mat, b, beta, y);  // argument-dependent lookup
}

}  // namespace SparseMatrixLib
