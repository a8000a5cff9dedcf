// SELL_C_Sigma.h — spMtxSELL_C_Sigma<ValT> of the RVVLASparse API
// (include/SELL_C_Sigma.h:23-101 of the reference): slices of C rows sorted by
// length inside windows of Sigma rows; slice i has height vBs[i], width
// vCl[i], starts at vCs[i] and holds sorted rows from vSBs[i]; element (k, j)
// of a slice at vCs[i] + j*vBs[i] + k; vPerm[sorted row] = original row.
#pragma once
#include <cstdint>
#include <vector>

#include "CRS.h"
#include "convert.h"
#include "rvvla_decl.h"

namespace SparseMatrixLib {

template <typename ValT>
class spMtxSELL_C_Sigma {
 public:
  size_t m = 0;
  size_t n = 0;
  size_t cnt_b = 0;
  size_t nz = 0;
  int C = 0;
  int Sigma = 0;
  std::vector<int> vCl;
  std::vector<int> vCs;
  std::vector<int> vBs;
  std::vector<int> vSBs;
  std::vector<uint32_t> vCol;
  std::vector<uint32_t> vPerm;
  std::vector<ValT> vVal;
  std::vector<int> vPartition;
  rvvla_dropin::MirrorSlot rvvla_dev;

  spMtxSELL_C_Sigma() {}
};

RVVLA_DROPIN_DECLARE_SPMV(spMtxSELL_C_Sigma)
RVVLA_DROPIN_DECLARE_SPMV_MIXED(spMtxSELL_C_Sigma)
RVVLA_DROPIN_DECLARE_CONVERT(spMtxSELL_C_Sigma)
RVVLA_DROPIN_DECLARE_TUNE(spMtxSELL_C_Sigma)

}  // namespace SparseMatrixLib
