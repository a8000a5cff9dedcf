// VHCC.h — spMtxVHCC<ValT> of the RVVLASparse API (include/VHCC.h:15-115 of
// the reference): nonzeros packed in vectors of vec_size, the ids of vectors
// holding row ends (veceor_ptr), per end-of-row vector log2(vec_size) scan
// masks plus one write mask (scan_mask), destination rows (row_arr) and one
// thr_info_t per thread.  On the GPU vec_size is 32 and there is one panel.
#pragma once
#include <cmath>
#include <cstdint>
#include <vector>

#include "CRS.h"
#include "convert.h"
#include "rvvla_decl.h"

namespace SparseMatrixLib {

struct vhcc_params {
  size_t num_threads;
  size_t num_panels;
  size_t tile_row;
  size_t tile_col;
  size_t vec_size;
  size_t n_masks;
  vhcc_params(size_t nt = 1, size_t np = 1, size_t row_tile = 512, size_t col_tile = 512, size_t vec = 8)
      : num_threads(nt), num_panels(np), tile_row(row_tile), tile_col(col_tile), vec_size(vec),
        n_masks((size_t)std::log2((double)vec)) {}
};

struct thr_info_t {
  int vbase;
  int rbase;
  int sbase;
  int last_row;
  int overflow_row;
  int start_vec;
  int end_vec;
  int panel_id;
  int merge_start;
  int merge_end;
};

typedef uint32_t index_t;

template <typename ValT>
class spMtxVHCC {
 public:
  size_t _num_rows = 0;
  size_t _num_cols = 0;
  size_t _num_entries = 0;
  size_t _num_vectors = 0;
  size_t _nnz_per_panel = 0;
  size_t _pad_entries = 0;
  size_t _extended_rows = 0;
  size_t _pad_rows = 0;
  std::vector<thr_info_t> _thr_info;
  std::vector<uint32_t> _veceor_ptr;
  std::vector<uint8_t> _scan_mask;
  std::vector<uint32_t> _row_arr;
  std::vector<uint32_t> _col_arr;
  std::vector<ValT> _vals_arr;
  vhcc_params params;
  rvvla_dropin::MirrorSlot rvvla_dev;

  spMtxVHCC() {}

  size_t get_n_masks() const { return params.n_masks; }
  int get_pad_rows() const { return (int)_pad_rows; }
  const thr_info_t* get_thr_info() const { return _thr_info.data(); }
  const uint32_t* get_veceor_ptr() const { return _veceor_ptr.data(); }
  const uint8_t* get_scan_mask() const { return _scan_mask.data(); }
  const uint32_t* get_row_arr() const { return _row_arr.data(); }
  const uint32_t* get_col_arr() const { return _col_arr.data(); }
  const ValT* get_vals_arr() const { return _vals_arr.data(); }
  vhcc_params get_params() const { return params; }
  std::vector<thr_info_t>& get_thr_info_reference() { return _thr_info; }
  std::vector<uint32_t>& get_veceor_reference() { return _veceor_ptr; }
  std::vector<uint8_t>& get_scan_mask_reference() { return _scan_mask; }
  std::vector<uint32_t>& get_row_arr_reference() { return _row_arr; }
  std::vector<uint32_t>& get_col_arr_reference() { return _col_arr; }
  std::vector<ValT>& get_vals_arr_reference() { return _vals_arr; }

  void freeMem() {
    _thr_info.clear(); _thr_info.shrink_to_fit();
    _veceor_ptr.clear(); _veceor_ptr.shrink_to_fit();
    _scan_mask.clear(); _scan_mask.shrink_to_fit();
    _row_arr.clear(); _row_arr.shrink_to_fit();
    _col_arr.clear(); _col_arr.shrink_to_fit();
    _vals_arr.clear(); _vals_arr.shrink_to_fit();
    rvvla_dev.reset();
  }
  ~spMtxVHCC() { freeMem(); }
  void set_params(const vhcc_params& info) { params = info; }
  void set_properties(size_t rows, size_t cols, size_t entries, size_t vectors, size_t pad_entries, size_t pad_rows) {
    _num_rows = rows;
    _num_cols = cols;
    _num_entries = entries;
    _num_vectors = vectors;
    _pad_entries = pad_entries;
    _pad_rows = pad_rows;
  }
};

RVVLA_DROPIN_DECLARE_SPMV(spMtxVHCC)
RVVLA_DROPIN_DECLARE_CONVERT(spMtxVHCC)
RVVLA_DROPIN_DECLARE_TUNE(spMtxVHCC)

}  // namespace SparseMatrixLib
