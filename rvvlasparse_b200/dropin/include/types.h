// types.h — status, operation and stage types of the RVVLASparse API
// (include/types.h:19-38 of the reference), for the GPU drop-in.
#pragma once
#include <stdint.h>

#include <iostream>

namespace SparseMatrixLib {

struct sparse_matrix_status {
  int code = 0;  // 0 = success; otherwise an rvvla_status from the GPU library
};

enum sparse_operation_t { SPARSE_OPERATION_NON_TRANSPOSE, SPARSE_OPERATION_TRANSPOSE };

struct sparse_matrix_descr {};

enum sparse_matrix_mv_stage {
  SPARSE_MATRIX_MV_PREPARATION,
  SPARSE_MATRIX_MV_MULT,
  SPARSE_MATRIX_MV_GET_RESULTS,
  SPARSE_MATRIX_MV_ALL_STAGES
};

}  // namespace SparseMatrixLib
