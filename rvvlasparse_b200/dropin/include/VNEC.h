// VNEC.h — spMtxVNEC<ValT> of the RVVLASparse API (include/VNEC.h:78-324 of
// the reference).  As there, the object is built from a CRS matrix that must
// outlive it (G is a non-owning pointer; M views G's arrays), the variant is
// chosen by IRD and the row count (L if m >= 2,000,000, else D if IRD >= the
// threshold, else S), and it cannot be copied, only moved.  Here the
// constructor builds the variant's structures on the GPU (NUM_THREADS_VNEC
// GPU threads, 2048 merge items each by default): the host pointers of the
// reference's per-thread structures stay null, their device copies live in
// the object's device mirror.
#pragma once
#include <type_traits>

#include "CRS.h"
#include "rvvla_decl.h"
#include "SpB_mxv_VNEC.h"

namespace SparseMatrixLib {

template <typename ValT>
class spMtxVNEC;

template <class V>
void rvvla_vnec_init(spMtxVNEC<V>& A, int nthreads);

template <typename ValT>
class spMtxVNEC {
 public:
  struct SpB_Matrix {
    int row = 0;
    int col = 0;
    int nnz = 0;
    int ptr_len = 0;
    int* ptr = nullptr;
    int* indices = nullptr;
    ValT* val = nullptr;
  };

  int NUM_THREADS_VNEC = 0;
  const spMtxCRS<ValT>* G = nullptr;
  SpB_Matrix M;
  coord* thread_coord_start = nullptr;
  coord* thread_coord_end = nullptr;
  int* ecr_indices = nullptr;
  int* NEC_NUM = nullptr;
  int** use_x_indices = nullptr;
  ValT** ecr_xx_val = nullptr;
  int* v_row_ptr = nullptr;
  int* col_start = nullptr;
  ValT* val_align = nullptr;
  int* spvv_len = nullptr;
  int** tasks = nullptr;
  int num_merge_items = 0;
  int items_per_thread = 0;
  int* diagonal_start = nullptr;
  int* diagonal_end = nullptr;
  int* nz_indices = nullptr;
  float IRD_mat = 0.f;
  SpB_VNEC_type vnec_t = SpB_VNEC_L;
  rvvla_dropin::MirrorSlot rvvla_dev;

  spMtxVNEC() {}
  // nthreads <= 0: one GPU thread per 2048 merge items (nonzeros + rows)
  explicit spMtxVNEC(const spMtxCRS<ValT>& G_, int nthreads = 0) : G(&G_) {
    view();
    rvvla_vnec_init(*this, nthreads);
  }
  spMtxVNEC(const spMtxVNEC&) = delete;
  spMtxVNEC& operator=(const spMtxVNEC&) = delete;
  spMtxVNEC(spMtxVNEC&& o)
      : NUM_THREADS_VNEC(o.NUM_THREADS_VNEC), G(o.G), num_merge_items(o.num_merge_items),
        items_per_thread(o.items_per_thread), IRD_mat(o.IRD_mat), vnec_t(o.vnec_t), rvvla_dev(std::move(o.rvvla_dev)) {
    o.G = nullptr;
    view();
  }
  spMtxVNEC& operator=(spMtxVNEC&& o) {
    NUM_THREADS_VNEC = o.NUM_THREADS_VNEC;
    G = o.G;
    o.G = nullptr;
    num_merge_items = o.num_merge_items;
    items_per_thread = o.items_per_thread;
    IRD_mat = o.IRD_mat;
    vnec_t = o.vnec_t;
    rvvla_dev = std::move(o.rvvla_dev);
    view();
    return *this;
  }
  void freeMem() { rvvla_dev.reset(); }
  ~spMtxVNEC() { freeMem(); }

 private:
  void view() {
    if (!G) return;
    M.row = (int)G->m;
    M.col = (int)G->n;
    M.nnz = (int)G->nz;
    M.ptr_len = (int)G->m + 1;
    M.ptr = G->Rst;
    M.indices = G->Col;
    M.val = G->Val;
  }
};

RVVLA_DROPIN_DECLARE_SPMV(spMtxVNEC)

}  // namespace SparseMatrixLib
