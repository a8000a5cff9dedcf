// rvv_shim.cpp — test infrastructure only (oracle side).
//
// extern "C" wrappers around the reference's UNMODIFIED RVV-only kernels
// (RVVLASparse src/rvv/spmv_mtx_csr5.cpp, src/rvv/spmv_mtx_vnec.cpp,
// src/rvv/spmv_vhcc.cpp), compiled from their own sources for x86-64 by
// oracle/Makefile target `ref-rvv` against the scalar intrinsic stand-in
// oracle/rvv_emul/riscv_vector.h (VLEN 256) into oracle/_ref/libref_rvv.so.
// Tests use them to pin the oracle's restatements of these three kernels to
// the reference's own code; nothing in the product path links this file.
//
// CSR5 and VHCC have no builder in the reference (asCSR5 is declared in
// include/CSR5.h:61-65 and never defined; VHCC has only setters,
// include/VHCC.h:80-112), so their objects are filled from layouts the
// oracle's builders produced.  VNEC is built by the reference's own
// constructor spMtxVNEC(const spMtxCRS&) (include/VNEC.h:200-227), which
// also picks the variant (D, S or L).  Every call goes through the
// reference's explicit specialisation sparse_mv<T, Fmt, true, stage>.
#include "riscv_vector.h"
#include "sparse_matrix.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <exception>
#include <string>
#include <vector>
#include <omp.h>

using namespace SparseMatrixLib;

namespace {

thread_local std::string g_last_error;

template <class M, class T>
struct Box {
  M A;
  std::vector<T> b, y;
};

template <class T>
struct VnecBox {
  spMtxCRS<T> G;
  spMtxVNEC<T>* A = nullptr;
  std::vector<T> b, y;
  ~VnecBox() { delete A; }
};

template <class T, class M, class Fn>
int run(M& box, T alpha, const T* b, T beta, T* y, Fn&& call) {
  try {
    std::memcpy(box.b.data(), b, box.b.size() * sizeof(T));
    std::memcpy(box.y.data(), y, box.y.size() * sizeof(T));
    const sparse_matrix_status st = call(alpha, beta);
    std::memcpy(y, box.y.data(), box.y.size() * sizeof(T));
    return st.code;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return -1;
  }
}

}  // namespace

extern "C" {

const char* refv_last_error() { return g_last_error.c_str(); }

// Known answers for the intrinsic stand-in (values worked out by hand from the
// RVV 1.0 intrinsic definitions); returns 0, or the number of the first check
// that failed.
int refv_selftest() {
  int k = 0;
#define REFV_CHECK(cond) \
  do {                   \
    ++k;                 \
    if (!(cond)) return k; \
  } while (0)
  // VLMAX at VLEN 256
  REFV_CHECK(__riscv_vsetvlmax_e64m2() == 8 && __riscv_vsetvlmax_e32m2() == 16 &&
             __riscv_vsetvlmax_e64m8() == 32 && __riscv_vsetvl_e64m2(5) == 5 && __riscv_vsetvl_e64m2(50) == 8);
  // mask bit i = bit i of the register image, LSB first
  const uint8_t bytes[32] = {0x05, 0x80};
  vbool32_t m = __riscv_vreinterpret_v_u8m1_b32(__riscv_vle8_v_u8m1(bytes, 2));
  REFV_CHECK(m.e[0] == 1 && m.e[1] == 0 && m.e[2] == 1 && m.e[7] == 0 && __riscv_vcpop_m_b32(m, 8) == 2);
  // viota: set elements below i
  vuint32m1_t io = __riscv_viota_m_u32m1(m, 8);
  REFV_CHECK(io.e[0] == 0 && io.e[1] == 1 && io.e[2] == 1 && io.e[3] == 2 && io.e[7] == 2);
  // vcompress packs the active elements to the front
  const double v8[8] = {10, 11, 12, 13, 14, 15, 16, 17};
  vfloat64m2_t a = __riscv_vle64_v_f64m2(v8, 8);
  vfloat64m2_t c = __riscv_vcompress_vm_f64m2(a, m, 8);
  REFV_CHECK(c.e[0] == 10 && c.e[1] == 12);
  // slides
  vfloat64m2_t d = __riscv_vfslide1down_vf_f64m2(a, -1.0, 8);
  REFV_CHECK(d.e[0] == 11 && d.e[6] == 17 && d.e[7] == -1);
  vfloat64m2_t u = __riscv_vslideup_vx_f64m2(__riscv_vfmv_v_f_f64m2(0.0, 8), a, 3, 8);
  REFV_CHECK(u.e[2] == 0 && u.e[3] == 10 && u.e[7] == 14);
  // gather: an index at or past VLMAX reads 0
  const uint32_t gi32[8] = {7, 0, 8, 1, 100, 2, 3, 4};
  vuint64m2_t gi = __riscv_vwcvtu_x_x_v_u64m2(__riscv_vle32_v_u32m1(gi32, 8), 8);
  vfloat64m2_t gth = __riscv_vrgather_vv_f64m2(a, gi, 8);
  REFV_CHECK(gth.e[0] == 17 && gth.e[1] == 10 && gth.e[2] == 0 && gth.e[4] == 0 && gth.e[7] == 14);
  // masked-undisturbed add keeps maskedoff where the mask is 0
  vfloat64m2_t off = __riscv_vfmv_v_f_f64m2(-5.0, 8);
  vfloat64m2_t mu = __riscv_vfadd_vv_f64m2_mu(m, off, a, a, 8);
  REFV_CHECK(mu.e[0] == 20 && mu.e[1] == -5 && mu.e[2] == 24 && mu.e[3] == -5);
  // vfmacc is fused: (1 + 2^-30)^2 - (1 + 2^-29) keeps the 2^-60 term
  const double e = 1.0 + std::ldexp(1.0, -30);
  vfloat64m2_t acc = __riscv_vfmv_v_f_f64m2(-(1.0 + std::ldexp(1.0, -29)), 1);
  acc = __riscv_vfmacc_vf_f64m2(acc, e, __riscv_vfmv_v_f_f64m2(e, 1), 1);
  REFV_CHECK(acc.e[0] == std::ldexp(1.0, -60));
  // reductions start from the scalar operand's element 0
  vfloat64m1_t s0 = __riscv_vfmv_v_f_f64m1(100.0, 1);
  REFV_CHECK(__riscv_vfmv_f_s_f64m1_f64(__riscv_vfredusum_vs_f64m2_f64m1(a, s0, 8)) == 100 + 108);
  // indexed loads take byte offsets; a vl above VLMAX acts as VLMAX
  const uint32_t boff[8] = {8, 0, 56, 16, 0, 0, 0, 0};
  vfloat64m2_t ix = __riscv_vloxei32_v_f64m2(v8, __riscv_vle32_v_u32m1(boff, 4), 4);
  REFV_CHECK(ix.e[0] == 11 && ix.e[1] == 10 && ix.e[2] == 17 && ix.e[3] == 12);
  vfloat64m1_t cl = __riscv_vfmv_v_f_f64m1(3.0, 64);
  REFV_CHECK(cl.e[0] == 3 && cl.e[3] == 3);
  // unsigned compare, masked integer add
  vuint32m1_t p = __riscv_vle32_v_u32m1(gi32, 8);
  vbool32_t le = __riscv_vmsleu_vv_u32m1_b32(p, __riscv_vmv_v_x_u32m1(7, 8), 8);
  REFV_CHECK(le.e[0] == 1 && le.e[2] == 0 && le.e[4] == 0 && __riscv_vcpop_m_b32(le, 8) == 6);
  vuint32m1_t pa = __riscv_vadd_vx_u32m1_mu(le, p, p, 1000u, 8);
  REFV_CHECK(pa.e[0] == 1007 && pa.e[2] == 8 && pa.e[4] == 100);
#undef REFV_CHECK
  return 0;
}
int refv_num_threads() { return omp_get_max_threads(); }
int refv_vlen() { return RVV_EMUL_VLEN; }

// ---------------------------------------------------------------- CSR5
// ints[0..10] = m, n, nnz, bit_y_offset, bit_seg_offset, tile_desc_len,
//               tail_tile_start, p, omega, sigma, num_offsets
// lens[0..5]  = |csr_row_pointer|, |csr_column_index| (= |csr_value|),
//               |tile_pointer|, |tile_descriptor|, |tile_empty_offset_pointer|,
//               |tile_empty_offset|
#define REFV_CSR5(VT, S)                                                                      \
  void* refv_csr5_new_##S(const int64_t* ints, const int64_t* lens, const int* row_ptr,       \
                          const uint32_t* col, const VT* val, const uint32_t* tile_ptr,       \
                          const uint32_t* tile_desc, const uint32_t* teo_ptr,                 \
                          const uint32_t* teo) {                                              \
    auto* box = new Box<spMtxCSR5<VT>, VT>();                                                 \
    auto& A = box->A;                                                                         \
    A._m = (int)ints[0]; A._n = (int)ints[1]; A._nnz = (int)ints[2];                          \
    A._bit_y_offset = (int)ints[3]; A._bit_seg_offset = (int)ints[4];                         \
    A._tile_desc_len = (int)ints[5]; A._tail_tile_start = (int)ints[6]; A._p = (int)ints[7];  \
    A._omega = (int)ints[8]; A._sigma = (int)ints[9]; A._num_offsets = (int)ints[10];         \
    A._csr_row_pointer.assign(row_ptr, row_ptr + lens[0]);                                    \
    A._csr_column_index.assign(col, col + lens[1]);                                           \
    A._csr_value.assign(val, val + lens[1]);                                                  \
    A._csr5_tile_pointer.assign(tile_ptr, tile_ptr + lens[2]);                                \
    A._csr5_tile_descriptor.assign(tile_desc, tile_desc + lens[3]);                           \
    A._csr5_tile_empty_offset_pointer.assign(teo_ptr, teo_ptr + lens[4]);                     \
    A._csr5_tile_empty_offset.assign(teo, teo + lens[5]);                                     \
    /* one cache line per OpenMP thread (the kernel clears and indexes it that way) */        \
    A._temp_calibrator.assign((size_t)omp_get_max_threads() * CSR5_CACHELINE / sizeof(VT),    \
                              VT(0));                                                         \
    box->b.assign((size_t)A._n, VT(0));                                                       \
    box->y.assign((size_t)A._m, VT(0));                                                       \
    return box;                                                                               \
  }                                                                                           \
  void refv_csr5_free_##S(void* h) { delete (Box<spMtxCSR5<VT>, VT>*)h; }                     \
  /* threads > 0: the default OpenMP team size for the call (the kernel sizes its */         \
  /* tile split and calibrator by omp_get_max_threads()).                          */         \
  int refv_csr5_spmv_##S(void* h, int threads, VT alpha, const VT* b, VT beta, VT* y) {       \
    auto& box = *(Box<spMtxCSR5<VT>, VT>*)h;                                                  \
    const int saved = omp_get_max_threads();                                                  \
    if (threads > 0) omp_set_num_threads(threads);                                            \
    if ((size_t)omp_get_max_threads() * CSR5_CACHELINE / sizeof(VT) >                         \
        box.A._temp_calibrator.size())                                                        \
      box.A._temp_calibrator.assign((size_t)omp_get_max_threads() * CSR5_CACHELINE /          \
                                    sizeof(VT), VT(0));                                       \
    const int rc = run(box, alpha, b, beta, y, [&](VT a, VT be) {                             \
      return sparse_mv<VT, spMtxCSR5, true>(SPARSE_OPERATION_NON_TRANSPOSE, a, box.A,         \
                                            sparse_matrix_descr{}, box.b, be, box.y);         \
    });                                                                                       \
    omp_set_num_threads(saved);                                                               \
    return rc;                                                                                \
  }
REFV_CSR5(double, f64)
REFV_CSR5(float, f32)

// ---------------------------------------------------------------- VHCC
// ints[0..7] = num_rows, num_cols, num_entries, num_vectors, pad_entries,
//              pad_rows, num_threads, vec_size
// lens[0..4] = |thr_info| (ints, 10 per thread), |veceor_ptr|,
//              |scan_mask| (bytes), |row_arr|, |col_arr| (= |vals_arr|)
#define REFV_VHCC(VT, S)                                                                      \
  void* refv_vhcc_new_##S(const int64_t* ints, const int64_t* lens, const int32_t* thr,       \
                          const uint32_t* veceor, const uint8_t* scan_mask,                   \
                          const uint32_t* row_arr, const uint32_t* col_arr, const VT* vals) { \
    auto* box = new Box<spMtxVHCC<VT>, VT>();                                                 \
    auto& A = box->A;                                                                         \
    A.set_params(vhcc_params((size_t)ints[6], 1, 512, 512, (size_t)ints[7]));                 \
    A.set_properties((size_t)ints[0], (size_t)ints[1], (size_t)ints[2], (size_t)ints[3],      \
                     (size_t)ints[4], (size_t)ints[5]);                                       \
    auto& ti = A.get_thr_info_reference();                                                    \
    ti.resize((size_t)lens[0] / 10);                                                          \
    static_assert(sizeof(thr_info_t) == 10 * sizeof(int32_t), "thr_info_t layout");           \
    if (!ti.empty()) std::memcpy(ti.data(), thr, ti.size() * sizeof(thr_info_t));             \
    A.get_veceor_reference().assign(veceor, veceor + lens[1]);                                \
    A.get_scan_mask_reference().assign(scan_mask, scan_mask + lens[2]);                       \
    A.get_row_arr_reference().assign(row_arr, row_arr + lens[3]);                             \
    A.get_col_arr_reference().assign(col_arr, col_arr + lens[4]);                             \
    A.get_vals_arr_reference().assign(vals, vals + lens[4]);                                  \
    box->b.assign((size_t)ints[1], VT(0));                                                    \
    box->y.assign((size_t)ints[0], VT(0));                                                    \
    return box;                                                                               \
  }                                                                                           \
  void refv_vhcc_free_##S(void* h) { delete (Box<spMtxVHCC<VT>, VT>*)h; }                     \
  /* The fp64 alpha = 1, beta = 0 branch copies tmp_y to y in a parallel region */          \
  /* of the default team size (src/rvv/spmv_vhcc.cpp:385) while it splits y by    */          \
  /* vhcc_params.num_threads, so a larger default team writes past y: the default */          \
  /* team size is set to the structure's thread count around the call, the setting */         \
  /* the reference is run with (OMP_NUM_THREADS = num_threads).                    */         \
  int refv_vhcc_spmv_##S(void* h, VT alpha, const VT* b, VT beta, VT* y) {                    \
    auto& box = *(Box<spMtxVHCC<VT>, VT>*)h;                                                  \
    const int saved = omp_get_max_threads();                                                  \
    omp_set_num_threads((int)box.A.get_params().num_threads);                                 \
    const int rc = run(box, alpha, b, beta, y, [&](VT a, VT be) {                             \
      return sparse_mv<VT, spMtxVHCC, true>(SPARSE_OPERATION_NON_TRANSPOSE, a, box.A,         \
                                            sparse_matrix_descr{}, box.b, be, box.y);         \
    });                                                                                       \
    omp_set_num_threads(saved);                                                               \
    return rc;                                                                                \
  }
REFV_VHCC(double, f64)
REFV_VHCC(float, f32)

// ---------------------------------------------------------------- VNEC
// info[0..1] = vnec_t (0 D, 1 S, 2 L), NUM_THREADS_VNEC; *ird = IRD_mat
#define REFV_VNEC(VT, S)                                                                      \
  /* threads > 0: the OpenMP team size while the constructor runs (it sets    */           \
  /* NUM_THREADS_VNEC from it and computes IRD with that many threads).       */           \
  void* refv_vnec_new_##S(int64_t m, int64_t n, int64_t nz, const int* Rst, const int* Col,   \
                          const VT* Val, int threads) {                                       \
    try {                                                                                     \
      auto* box = new VnecBox<VT>();                                                          \
      box->G = spMtxCRS<VT>((size_t)m, (size_t)n, (size_t)nz, Rst, Col, Val);                 \
      const int saved = omp_get_max_threads();                                                \
      if (threads > 0) omp_set_num_threads(threads);                                          \
      box->A = new spMtxVNEC<VT>(box->G);                                                     \
      omp_set_num_threads(saved);                                                             \
      box->b.assign((size_t)n, VT(0));                                                        \
      box->y.assign((size_t)m, VT(0));                                                        \
      return box;                                                                             \
    } catch (const std::exception& e) {                                                       \
      g_last_error = e.what();                                                                \
      return nullptr;                                                                         \
    }                                                                                         \
  }                                                                                           \
  void refv_vnec_free_##S(void* h) { delete (VnecBox<VT>*)h; }                                \
  void refv_vnec_info_##S(void* h, int64_t* info, double* ird) {                              \
    auto& box = *(VnecBox<VT>*)h;                                                             \
    info[0] = (int64_t)box.A->vnec_t;                                                         \
    info[1] = (int64_t)box.A->NUM_THREADS_VNEC;                                               \
    *ird = (double)box.A->IRD_mat;                                                            \
  }                                                                                           \
  int refv_vnec_spmv_##S(void* h, VT alpha, const VT* b, VT beta, VT* y) {                    \
    auto& box = *(VnecBox<VT>*)h;                                                             \
    return run(box, alpha, b, beta, y, [&](VT a, VT be) {                                     \
      return sparse_mv<VT, spMtxVNEC, true>(SPARSE_OPERATION_NON_TRANSPOSE, a, *box.A,        \
                                            sparse_matrix_descr{}, box.b, be, box.y);         \
    });                                                                                       \
  }
REFV_VNEC(double, f64)
REFV_VNEC(float, f32)

// The reference's VNEC kernels read structures that no reference code fills
// (the constructor computes only IRD and the variant): this sets them from a
// layout the oracle's VNEC builder made for the same matrix, allocated the way
// the reference's freeMem() releases them (include/VNEC.h:265-319: malloc'd
// arrays, NUM_THREADS_VNEC + 1 slots for use_x_indices / ecr_xx_val, one
// malloc'd row list per thread in tasks), then selects the variant.
// ints[0..1] = vnec_t (0 D, 1 S, 2 L), NUM_THREADS_VNEC (<= 256, the D and L
//              kernels' carry arrays)
// lens[0..7] = |ecr_indices|, |use_x_indices|, |v_row_ptr|, |col_start|,
//              |val_align|, |tasks|, |row_begin| (= |row_end|), |reorder_col|
// Arrays a variant does not use may be NULL (their lengths 0).
}  // extern "C"
namespace {
template <class T>
T* dup(const T* src, int64_t n, int64_t pad = 0) {
  T* p = (T*)std::calloc((size_t)(n + pad > 0 ? n + pad : 1), sizeof(T));
  if (p && src && n > 0) std::memcpy(p, src, (size_t)n * sizeof(T));
  return p;
}
}  // namespace
extern "C" {
#define REFV_VNEC_FILL(VT, S)                                                                 \
  int refv_vnec_fill_##S(void* h, const int64_t* ints, const int64_t* lens, const int* tcs,    \
                         const int* tce, const int* nec, const int* ux_ptr, const int* ux,     \
                         const int* ecr, const int* vrp, const int* cs, const VT* va,          \
                         const int* tasks, const int* ts, const int* te, const int* sv,        \
                         const int* rb, const int* re, const int* rc, const VT* rv) {          \
    auto& A = *((VnecBox<VT>*)h)->A;                                                          \
    const int NT = (int)ints[1];                                                              \
    if (NT < 1 || NT > 256 || ints[0] < 0 || ints[0] > 2) {                                   \
      g_last_error = "refv_vnec_fill: bad variant or thread count";                            \
      return -1;                                                                              \
    }                                                                                         \
    A.freeMem();                                                                              \
    A.NUM_THREADS_VNEC = NT;                                                                  \
    A.vnec_t = (SpB_VNEC_type)ints[0];                                                        \
    A.thread_coord_start = (coord*)dup(tcs, 2 * (int64_t)NT);                                 \
    A.thread_coord_end = (coord*)dup(tce, 2 * (int64_t)NT);                                   \
    const int64_t nl = std::is_same<VT, float>::value ? nLanes_f32 : nLanes_f64;              \
    if (nec) {                                                                                \
      A.NEC_NUM = dup(nec, NT);                                                               \
      A.use_x_indices = (int**)std::calloc((size_t)NT + 1, sizeof(int*));                     \
      A.ecr_xx_val = (VT**)std::calloc((size_t)NT + 1, sizeof(VT*));                          \
      for (int t = 0; t < NT; ++t) {                                                          \
        A.use_x_indices[t] = dup(ux + ux_ptr[t], (int64_t)nec[t], nl);                        \
        A.ecr_xx_val[t] = dup<VT>(nullptr, (int64_t)nec[t], nl);                              \
      }                                                                                       \
    }                                                                                         \
    if (ecr) A.ecr_indices = dup(ecr, lens[0]);                                               \
    if (vrp) A.v_row_ptr = dup(vrp, lens[2]);                                                 \
    if (cs) A.col_start = dup(cs, lens[3]);                                                   \
    if (va) A.val_align = dup(va, lens[4]);                                                   \
    if (tasks) {                                                                              \
      A.tasks = (int**)std::calloc((size_t)NT, sizeof(int*));                                 \
      for (int t = 0; t < NT; ++t) {                                                          \
        const int64_t cnt = std::max<int64_t>((int64_t)te[t] - ts[t], (int64_t)sv[t]);        \
        const int64_t avail = std::max<int64_t>(0, std::min<int64_t>(cnt, lens[5] - ts[t]));  \
        A.tasks[t] = dup(tasks + ts[t], avail, cnt - avail + nl);                             \
      }                                                                                       \
      A.spvv_len = dup(sv, NT);                                                               \
      A.reorder_mat.task_start = dup(ts, NT);                                                 \
      A.reorder_mat.task_end = dup(te, NT);                                                   \
      A.reorder_mat.row_begin = dup(rb, lens[6], nl);                                         \
      A.reorder_mat.row_end = dup(re, lens[6], nl);                                           \
      A.reorder_mat.col = dup(rc, lens[7], nl);                                               \
      A.reorder_mat.nnz = dup(rv, lens[7], nl);                                               \
    }                                                                                         \
    return 0;                                                                                 \
  }
REFV_VNEC_FILL(double, f64)
REFV_VNEC_FILL(float, f32)

}  // extern "C"
