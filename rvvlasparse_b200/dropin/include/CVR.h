// CVR.h — spMtxCVR<ValT> of the RVVLASparse API (include/CVR.h:22-81 of the
// reference): SIMD_LEN lanes stream their rows' nonzeros (vPack_vec_vals /
// vPack_vec_cols); vPack_vec_record holds (position, row) pairs that flush a
// lane into y; writeback_pos_record holds per-thread blocks of SIMD_LEN + 2
// ints (first vector, first record, tail row of each lane).
#pragma once
#include <cstdint>
#include <vector>

#include "CRS.h"
#include "convert.h"
#include "rvvla_decl.h"

namespace SparseMatrixLib {

template <typename ValT>
class spMtxCVR {
 public:
  size_t nItems = 0;
  size_t numRows = 0;
  size_t numCols = 0;
  size_t SIMD_LEN = 1;
  int Nthreads = 1;
  int Nthreads_avail = 1;
  std::vector<ValT> vPack_vec_vals;
  std::vector<uint32_t> vPack_vec_cols;
  std::vector<int> vPack_vec_record;
  std::vector<int> writeback_pos_record;
  rvvla_dropin::MirrorSlot rvvla_dev;

  spMtxCVR() {}
  void freeMem() {
    vPack_vec_vals.clear(); vPack_vec_vals.shrink_to_fit();
    vPack_vec_cols.clear(); vPack_vec_cols.shrink_to_fit();
    vPack_vec_record.clear(); vPack_vec_record.shrink_to_fit();
    writeback_pos_record.clear(); writeback_pos_record.shrink_to_fit();
    rvvla_dev.reset();
  }
};

RVVLA_DROPIN_DECLARE_SPMV(spMtxCVR)
RVVLA_DROPIN_DECLARE_CONVERT(spMtxCVR)
RVVLA_DROPIN_DECLARE_TUNE(spMtxCVR)

}  // namespace SparseMatrixLib
