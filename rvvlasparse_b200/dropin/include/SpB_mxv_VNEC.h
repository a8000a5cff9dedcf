// SpB_mxv_VNEC.h — constants and enums of the VNEC format in the RVVLASparse
// API (include/SpB_mxv_VNEC.h:22-65 of the reference).
#pragma once
#include <cstddef>

#define nLanes_f32 16
#define nLanes_f64 8
#define IRD_thr_fp32 0.437
#define IRD_thr_fp64 0.477

namespace SparseMatrixLib {

typedef size_t SpB_Index;

enum SpB_VNEC_type { SpB_VNEC_D, SpB_VNEC_S, SpB_VNEC_L };

struct coord {
  int x;
  int y;
};

enum SpB_Type {
  SpB_NULL_TYPE,
  SpB_BOOL,
  SpB_INT8,
  SpB_INT16,
  SpB_INT32,
  SpB_INT64,
  SpB_UINT8,
  SpB_UINT16,
  SpB_UINT32,
  SpB_UINT64,
  SpB_FP32,
  SpB_FP64,
  SpB_Type_N
};

}  // namespace SparseMatrixLib
