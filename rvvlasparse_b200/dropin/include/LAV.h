// LAV.h — spMtxLAV<type> of the RVVLASparse API (include/LAV.h:10-94 of the
// reference): dense columns in segments of segment_len, rows in chunks of
// SIMD_Lanes (out_order), lane-major steps (val/col_id) with per-step active
// lane counts (mask), chunk offsets per segment, the rest in sparse_part.
#pragma once
#include <cstdint>
#include <vector>

#include "CRS.h"
#include "convert.h"
#include "rvvla_decl.h"

namespace SparseMatrixLib {

template <typename type>
struct spMtxLAV {
  size_t SIMD_Lanes = 8;
  int m = 0;
  int n = 0;
  int nz = 0;
  size_t segment_count = 0;
  size_t chunk_count = 0;
  double T = 0.2;
  int segment_len = 40000;
  std::vector<int> chunk_offsets;
  std::vector<int> chunk_offsets_full_mask;
  std::vector<size_t> segment_ptr;
  std::vector<uint32_t> out_order;
  std::vector<uint16_t> mask;
  std::vector<type> val;
  std::vector<uint32_t> col_id;
  spMtxCRS<type> sparse_part;
  rvvla_dropin::MirrorSlot rvvla_dev;

  spMtxLAV() {}
  void freeMem() {
    chunk_offsets.clear(); chunk_offsets.shrink_to_fit();
    chunk_offsets_full_mask.clear(); chunk_offsets_full_mask.shrink_to_fit();
    segment_ptr.clear(); segment_ptr.shrink_to_fit();
    out_order.clear(); out_order.shrink_to_fit();
    mask.clear(); mask.shrink_to_fit();
    val.clear(); val.shrink_to_fit();
    col_id.clear(); col_id.shrink_to_fit();
    sparse_part.freeMem();
    rvvla_dev.reset();
  }
};

RVVLA_DROPIN_DECLARE_SPMV(spMtxLAV)
RVVLA_DROPIN_DECLARE_CONVERT(spMtxLAV)
RVVLA_DROPIN_DECLARE_TUNE(spMtxLAV)

}  // namespace SparseMatrixLib
