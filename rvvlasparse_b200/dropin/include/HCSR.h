// HCSR.h — spMtxHCSR<ValT> of the RVVLASparse API (include/HCSR.h:20-114 of
// the reference): R x C blocks; block_ptr (nonzero offset per block),
// row_offset (bits 31:30 block kind 0 empty / 1 CSR / 2 COO, bits 29:0 offset
// into row_ptr), row_ptr, uint16 local columns, values.  Host vectors, plus
// the device copy used by the GPU drop-in.
#pragma once
#include <cstdint>
#include <vector>

#include "CRS.h"
#include "convert.h"
#include "rvvla_decl.h"

namespace SparseMatrixLib {

template <typename ValT>
struct inCRS {
  size_t m = 0;
  size_t n = 0;
  size_t nz = 0;
  std::vector<int> row_ptr;
  std::vector<int> col_idx;
  std::vector<ValT> values;
};

template <typename ValT>
class spMtxHCSR {
 public:
  size_t R = 0;
  size_t C = 0;
  size_t m = 0;
  size_t n = 0;
  size_t nz = 0;
  size_t b_m = 0;
  size_t b_n = 0;
  std::vector<int> block_ptr;
  std::vector<uint32_t> row_offset;
  std::vector<uint32_t> row_ptr;
  std::vector<uint16_t> col_idx;
  std::vector<ValT> values;
  rvvla_dropin::MirrorSlot rvvla_dev;

  spMtxHCSR() {}
  spMtxHCSR(size_t m_, size_t n_, size_t nz_, size_t R_, size_t C_)
      : R(R_), C(C_), m(m_), n(n_), nz(nz_), b_m((m_ + R_ - 1) / R_), b_n((n_ + C_ - 1) / C_) {}
};

RVVLA_DROPIN_DECLARE_SPMV(spMtxHCSR)
RVVLA_DROPIN_DECLARE_SPMV_MIXED(spMtxHCSR)
RVVLA_DROPIN_DECLARE_CONVERT(spMtxHCSR)
RVVLA_DROPIN_DECLARE_TUNE(spMtxHCSR)

}  // namespace SparseMatrixLib
