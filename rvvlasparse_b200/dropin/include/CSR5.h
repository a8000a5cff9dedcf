// CSR5.h — spMtxCSR5<ValT> of the RVVLASparse API (include/CSR5.h:28-112 of
// the reference): CSR plus p tiles of omega x sigma nonzeros (full tiles
// stored transposed), per-tile row pointers (bit 31 = the tile has empty
// rows), per-lane descriptors (y_offset / seg_offset / sigma bit-flags) and
// the empty-row offset maps.  On the GPU omega is 32 (a warp).
#pragma once
#include <cstdint>
#include <type_traits>
#include <vector>

#include "CRS.h"
#include "rvvla_decl.h"
#include "alignment_allocator.h"
#include "convert.h"

#define CSR5_SUCCESS 0
#define CSR5_UNKNOWN_FORMAT -1
#define CSR5_UNSUPPORTED_OMEGA -2
#define CSR5_CONVERTION_FAILED -3
#define CSR5_UNSUPPORTED_SPMV -4
#define CSR5_UNSUPPORTED_VALUE_TYPE -5

#define CSR5_FORMAT_CSR 0
#define CSR5_FORMAT_CSR5 1

#define CSR5_AVX2_OMEGA 4
#define CSR5_AVX2_SIGMA 4
#define CSR5_SCALAR_OMEGA 4
#define CSR5_SCALAR_SIGMA 4
#define CSR5_CACHELINE 64

namespace SparseMatrixLib {

template <typename T, typename U>
std::common_type_t<T, U> iceil(T num, U den) {
  return (num + den - 1) / den;
}

inline uint32_t remove_sign(uint32_t value) { return value & 0x7FFFFFFFu; }

template <class ValT>
class spMtxCSR5 {
 public:
  // Keeps a copy of the CSR arrays (format CSR).
  int inputCSR(int m, int n, int nnz, int* csr_row_pointer_ptr, int* csr_column_index_ptr, ValT* csr_value_ptr);
  // Builds the CSR5 layout on the GPU (params "omega" must be 32 if given,
  // "sigma" defaults to 16) and fills the fields below; CSR5_SUCCESS or a
  // CSR5_* error code.
  int asCSR5(const convertParams& params);

  int _m = 0;
  int _n = 0;
  int _nnz = 0;
  int _bit_y_offset = 0;
  int _bit_seg_offset = 0;
  int _tile_desc_len = 0;
  int _tail_tile_start = 0;
  int _p = 0;
  int _omega = 0;
  int _sigma = 0;

  std::vector<int, AlignmentAllocator<int, CSR5_CACHELINE>> _csr_row_pointer;
  std::vector<uint32_t, AlignmentAllocator<uint32_t, CSR5_CACHELINE>> _csr_column_index;
  std::vector<ValT, AlignmentAllocator<ValT, CSR5_CACHELINE>> _csr_value;
  std::vector<uint32_t, AlignmentAllocator<uint32_t, CSR5_CACHELINE>> _csr5_tile_pointer;
  std::vector<uint32_t, AlignmentAllocator<uint32_t, CSR5_CACHELINE>> _csr5_tile_descriptor;
  int _num_offsets = 0;
  std::vector<uint32_t, AlignmentAllocator<uint32_t, CSR5_CACHELINE>> _csr5_tile_empty_offset_pointer;
  std::vector<uint32_t, AlignmentAllocator<uint32_t, CSR5_CACHELINE>> _csr5_tile_empty_offset;
  std::vector<ValT, AlignmentAllocator<ValT, CSR5_CACHELINE>> _temp_calibrator;
  rvvla_dropin::MirrorSlot rvvla_dev;

  template <typename T, typename Allocator>
  void clearAndShrink(std::vector<T, Allocator>& vec) {
    vec.clear();
    vec.shrink_to_fit();
  }
  void freeMem() {
    clearAndShrink(_csr_row_pointer);
    clearAndShrink(_csr_column_index);
    clearAndShrink(_csr_value);
    clearAndShrink(_csr5_tile_pointer);
    clearAndShrink(_csr5_tile_descriptor);
    clearAndShrink(_csr5_tile_empty_offset_pointer);
    clearAndShrink(_csr5_tile_empty_offset);
    clearAndShrink(_temp_calibrator);
    rvvla_dev.reset();
  }
  ~spMtxCSR5() { freeMem(); }

  int format() const { return _format; }
  void rvvla_set_format(int f) { _format = f; }

 private:
  int _format = CSR5_FORMAT_CSR;
};

RVVLA_DROPIN_DECLARE_SPMV(spMtxCSR5)
RVVLA_DROPIN_DECLARE_SPMV_MIXED(spMtxCSR5)
RVVLA_DROPIN_DECLARE_CONVERT(spMtxCSR5)
RVVLA_DROPIN_DECLARE_TUNE(spMtxCSR5)

}  // namespace SparseMatrixLib
