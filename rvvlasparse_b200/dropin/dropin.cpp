// dropin.cpp — the RVVLASparse C++ API (sparse_mv / convert over the eight
// format classes, host std::vector data) on top of the GPU library's C ABI.
//
// Each matrix object carries a DeviceMirror: the device arrays and the C ABI
// descriptor of its format.  convert() builds on the GPU, copies the built
// arrays into the object's public host fields and keeps the device copy;
// sparse_mv() uploads the host fields only when the object has no mirror yet,
// then stages b (and y when it is read) through per-mirror device buffers.
// Library failures inside sparse_mv come back as sparse_matrix_status.code
// (an rvvla_status); convert throws like the reference's HCSR builder
// (src/scalar/crs_to_hcsr.cpp:38-91): std::invalid_argument, std::length_error,
// std::runtime_error.
#include <algorithm>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "rvvla.h"
#include "sparse_matrix.h"

namespace rvvla_dropin {

struct DeviceMirror {
  std::vector<void*> bufs;  // uploaded host arrays (rvvla_malloc)
  void* x = nullptr;        // staging for b
  size_t xbytes = 0;
  void* y = nullptr;        // staging for y
  size_t ybytes = 0;
  rvvla_crs crs{};
  rvvla_hcsr hcsr{};
  rvvla_sell sell{};
  rvvla_csr5 csr5{};
  rvvla_lav lav{};
  rvvla_vnec vnec{};
  rvvla_vhcc vhcc{};
  rvvla_cvr cvr{};
  // builder outputs (freed with the format's free function)
  rvvla_hcsr_owned ho{};
  rvvla_sell_owned so{};
  rvvla_csr5_owned co{};
  rvvla_lav_owned lo{};
  rvvla_vnec_owned vo{};
  rvvla_vhcc_owned wo{};
  rvvla_cvr_owned ro{};
  rvvla_transpose_owned to{};
  bool has_transpose = false;
  ~DeviceMirror() {
    for (void* p : bufs) rvvla_free(p);
    rvvla_free(x);
    rvvla_free(y);
    rvvla_hcsr_free(&ho);
    rvvla_sell_free(&so);
    rvvla_csr5_free(&co);
    rvvla_lav_free(&lo);
    rvvla_vnec_free(&vo);
    rvvla_vhcc_free(&wo);
    rvvla_cvr_free(&ro);
    rvvla_csr_transpose_free(&to);
  }
};

void release(DeviceMirror* m) { delete m; }

}  // namespace rvvla_dropin

namespace SparseMatrixLib {
namespace {

using rvvla_dropin::DeviceMirror;

struct StatusError : std::runtime_error {
  int code;
  StatusError(int c, const std::string& what) : std::runtime_error(what), code(c) {}
};

void check(int rc, const char* where) {
  if (rc != RVVLA_OK) throw StatusError(rc, std::string(where) + ": " + rvvla_last_error());
}

// convert() errors, typed like the reference builder's exceptions
[[noreturn]] void throw_build(int rc, const char* where) {
  const std::string msg = std::string(where) + ": " + rvvla_last_error();
  if (rc == RVVLA_ERR_INVALID_ARG) throw std::invalid_argument(msg);
  if (rc == RVVLA_ERR_TOO_LARGE) throw std::length_error(msg);
  throw std::runtime_error(msg);
}

template <class T>
int val_bytes() {
  return (int)sizeof(T);
}

template <class T>
const T* upload(DeviceMirror& M, const T* h, size_t n) {
  if (n == 0) return nullptr;
  void* p = nullptr;
  check(rvvla_malloc(&p, n * sizeof(T)), "rvvla_malloc");
  M.bufs.push_back(p);
  check(rvvla_memcpy(p, h, n * sizeof(T), nullptr), "rvvla_memcpy");
  return static_cast<const T*>(p);
}

template <class T, class A>
void download(std::vector<T, A>& h, const void* d, size_t n) {
  h.resize(n);
  if (n) check(rvvla_memcpy(h.data(), d, n * sizeof(T), nullptr), "rvvla_memcpy");
}

void ensure(void*& buf, size_t& have, size_t bytes) {
  if (have >= bytes) return;
  rvvla_free(buf);
  buf = nullptr;
  have = 0;
  check(rvvla_malloc(&buf, bytes), "rvvla_malloc");
  have = bytes;
}

template <class Mtx>
DeviceMirror& fresh_mirror(const Mtx& A) {
  A.rvvla_dev.set(new DeviceMirror());
  return *A.rvvla_dev.get();
}

int param_i(const convertParams& p, const char* k, int dflt) {
  auto it = p.param.find(k);
  return it == p.param.end() ? dflt : it->second.i;
}

double param_d(const convertParams& p, const char* k, double dflt) {
  auto it = p.param.find(k);
  return it == p.param.end() ? dflt : it->second.d;
}

// ------------------------------------------------------------------ CRS
template <class T>
DeviceMirror& crs_mirror(const spMtxCRS<T>& A) {
  if (A.rvvla_dev.get()) return *A.rvvla_dev.get();
  DeviceMirror& M = fresh_mirror(A);
  rvvla_crs& d = M.crs;
  d.m = (int64_t)A.m;
  d.n = (int64_t)A.n;
  d.nz = (int64_t)A.nz;
  d.Rst = upload(M, A.Rst, A.m + 1);
  d.Col = upload(M, A.Col, A.nz);
  d.Val = upload(M, A.Val, A.nz);
  if (A.m > 0) {
    const int dt = std::is_same<T, double>::value ? RVVLA_F64 : RVVLA_F32;
    const int64_t len = rvvla_crs_plan_len(d.m, d.nz, dt);
    void* plan = nullptr;
    check(rvvla_malloc(&plan, (size_t)std::max<int64_t>(len, 1) * sizeof(int32_t)), "rvvla_malloc");
    M.bufs.push_back(plan);
    int64_t tiles = 0;
    int32_t kind = 0;
    check(rvvla_crs_analyze(&d, dt, static_cast<int32_t*>(plan), &tiles, &kind, nullptr), "rvvla_crs_analyze");
    d.plan = static_cast<const int32_t*>(plan);
    d.plan_tiles = tiles;
    d.plan_kind = kind;
  }
  return M;
}

// b -> device, y -> device when it is read; call(x, y); y -> host
template <class T, class F>
sparse_matrix_status run(DeviceMirror& M, size_t m, size_t n, const std::vector<T>& b, T beta, std::vector<T>& y,
                         bool reads_y, F&& call) {
  sparse_matrix_status st;
  if (b.size() < n || y.size() < m) {
    st.code = RVVLA_ERR_INVALID_ARG;
    return st;
  }
  ensure(M.x, M.xbytes, std::max<size_t>(n, 1) * sizeof(T));
  ensure(M.y, M.ybytes, std::max<size_t>(m, 1) * sizeof(T));
  // the caller's vectors are pageable: staged through the library's
  // page-locked buffers, host copies overlapping the DMA
  if (n) check(rvvla_copy_h2d(M.x, b.data(), n * sizeof(T), nullptr), "rvvla_copy_h2d");
  if (m && (reads_y || beta != T(0))) check(rvvla_copy_h2d(M.y, y.data(), m * sizeof(T), nullptr), "rvvla_copy_h2d");
  st.code = call(static_cast<const T*>(M.x), static_cast<T*>(M.y));
  if (st.code == RVVLA_OK && m) check(rvvla_copy_d2h(y.data(), M.y, m * sizeof(T), nullptr), "rvvla_copy_d2h");
  return st;
}

template <class F>
sparse_matrix_status guarded(F&& f) {
  try {
    return f();
  } catch (const StatusError& e) {
    sparse_matrix_status st;
    st.code = e.code;
    return st;
  } catch (const std::bad_alloc&) {
    sparse_matrix_status st;
    st.code = RVVLA_ERR_CUDA;
    return st;
  }
}

bool multiplies(sparse_matrix_mv_stage s) { return s == SPARSE_MATRIX_MV_MULT || s == SPARSE_MATRIX_MV_ALL_STAGES; }

int crs_call(const rvvla_crs* d, double a, const double* x, double b, double* y) {
  return rvvla_crs_spmv_f64(d, a, x, b, y, nullptr);
}
int crs_call(const rvvla_crs* d, float a, const float* x, float b, float* y) {
  return rvvla_crs_spmv_f32(d, a, x, b, y, nullptr);
}

template <class T>
sparse_matrix_status crs_spmv(sparse_operation_t op, T alpha, const spMtxCRS<T>& A, const std::vector<T>& b, T beta,
                              std::vector<T>& y, sparse_matrix_mv_stage stage) {
  return guarded([&] {
    if (!multiplies(stage)) return sparse_matrix_status{};
    DeviceMirror& M = crs_mirror(A);
    if (op == SPARSE_OPERATION_TRANSPOSE) {
      // y = alpha * A^T b + beta * y through the transposed CRS (built once)
      if (!M.has_transpose) {
        check(rvvla_csr_transpose(&M.crs, val_bytes<T>(), &M.to, nullptr), "rvvla_csr_transpose");
        M.has_transpose = true;
      }
      return run<T>(M, A.n, A.m, b, beta, y, false, [&](const T* x, T* yy) {
        return std::is_same<T, double>::value
                   ? rvvla_spmv_adjoint_x_f64(&M.to.h, (double)alpha, (const double*)x, (double)beta, (double*)yy,
                                              nullptr)
                   : rvvla_spmv_adjoint_x_f32(&M.to.h, (float)alpha, (const float*)x, (float)beta, (float*)yy,
                                              nullptr);
      });
    }
    return run<T>(M, A.m, A.n, b, beta, y, false,
                  [&](const T* x, T* yy) { return crs_call(&M.crs, alpha, x, beta, yy); });
  });
}

// ------------------------------------------------------------------ HCSR
template <class T>
DeviceMirror& hcsr_mirror(const spMtxHCSR<T>& A) {
  if (A.rvvla_dev.get()) return *A.rvvla_dev.get();
  DeviceMirror& M = fresh_mirror(A);
  rvvla_hcsr& d = M.hcsr;
  d.R = (int64_t)A.R; d.C = (int64_t)A.C; d.m = (int64_t)A.m; d.n = (int64_t)A.n; d.nz = (int64_t)A.nz;
  d.b_m = (int64_t)A.b_m; d.b_n = (int64_t)A.b_n;
  d.block_ptr = upload(M, A.block_ptr.data(), A.block_ptr.size());
  d.row_offset = upload(M, A.row_offset.data(), A.row_offset.size());
  d.row_ptr = upload(M, A.row_ptr.data(), A.row_ptr.size());
  d.col_idx = upload(M, A.col_idx.data(), A.col_idx.size());
  d.values = upload(M, A.values.data(), A.values.size());
  d.row_ptr_len = (int64_t)A.row_ptr.size();
  return M;
}

template <class T>
void hcsr_convert(spMtxHCSR<T>& dist, const spMtxCRS<T>& src, const convertParams& p) {
  // defaults of convert<T, spMtxHCSR, false> (src/scalar/crs_to_hcsr.cpp:140-142, 157-159)
  const int dflt = std::is_same<T, double>::value ? 2000 : 4000;
  const int R = param_i(p, "R", dflt), C = param_i(p, "C", dflt);
  const double pp = param_d(p, "p", 2.0);
  if (R <= 0 || C <= 0) throw std::invalid_argument("crs_to_HCSR: R and C must be positive");
  DeviceMirror& S = crs_mirror(src);
  auto* M = new DeviceMirror();
  std::unique_ptr<DeviceMirror, void (*)(DeviceMirror*)> hold(M, rvvla_dropin::release);
  const int rc = rvvla_hcsr_build(&S.crs, val_bytes<T>(), R, C, pp, &M->ho, nullptr);
  if (rc) throw_build(rc, "convert<spMtxHCSR>");
  const rvvla_hcsr& h = M->ho.h;
  dist.R = (size_t)h.R; dist.C = (size_t)h.C; dist.m = (size_t)h.m; dist.n = (size_t)h.n; dist.nz = (size_t)h.nz;
  dist.b_m = (size_t)h.b_m; dist.b_n = (size_t)h.b_n;
  const size_t nb1 = (size_t)(h.b_m * h.b_n + 1);
  download(dist.block_ptr, h.block_ptr, nb1);
  download(dist.row_offset, h.row_offset, nb1);
  download(dist.row_ptr, h.row_ptr, (size_t)h.row_ptr_len);
  download(dist.col_idx, h.col_idx, (size_t)h.nz);
  download(dist.values, h.values, (size_t)h.nz);
  M->hcsr = h;
  dist.rvvla_dev.set(hold.release());
}

int hcsr_call(const rvvla_hcsr* d, double a, const double* x, double b, double* y) {
  return rvvla_hcsr_spmv_f64(d, a, x, b, y, nullptr);
}
int hcsr_call(const rvvla_hcsr* d, float a, const float* x, float b, float* y) {
  return rvvla_hcsr_spmv_f32(d, a, x, b, y, nullptr);
}

// ------------------------------------------------------------------ SELL
template <class T>
DeviceMirror& sell_mirror(const spMtxSELL_C_Sigma<T>& A) {
  if (A.rvvla_dev.get()) return *A.rvvla_dev.get();
  DeviceMirror& M = fresh_mirror(A);
  rvvla_sell& d = M.sell;
  d.m = (int64_t)A.m; d.n = (int64_t)A.n; d.cnt_b = (int64_t)A.cnt_b; d.nz = (int64_t)A.nz;
  d.C = A.C; d.Sigma = A.Sigma;
  d.vCl = upload(M, A.vCl.data(), A.vCl.size());
  d.vCs = upload(M, A.vCs.data(), A.vCs.size());
  d.vBs = upload(M, A.vBs.data(), A.vBs.size());
  d.vSBs = upload(M, A.vSBs.data(), A.vSBs.size());
  d.vCol = upload(M, A.vCol.data(), A.vCol.size());
  d.vPerm = upload(M, A.vPerm.data(), A.vPerm.size());
  d.vVal = upload(M, A.vVal.data(), A.vVal.size());
  d.len = (int64_t)A.vVal.size();
  return M;
}

template <class T>
void sell_convert(spMtxSELL_C_Sigma<T>& dist, const spMtxCRS<T>& src, const convertParams& p) {
  const int C = param_i(p, "C", 32);
  const int sigma = param_i(p, "Sigma", param_i(p, "sigma", 256));
  DeviceMirror& S = crs_mirror(src);
  auto* M = new DeviceMirror();
  std::unique_ptr<DeviceMirror, void (*)(DeviceMirror*)> hold(M, rvvla_dropin::release);
  const int rc = rvvla_sell_build(&S.crs, val_bytes<T>(), C, sigma, &M->so, nullptr);
  if (rc) throw_build(rc, "convert<spMtxSELL_C_Sigma>");
  const rvvla_sell& h = M->so.h;
  dist.m = (size_t)h.m; dist.n = (size_t)h.n; dist.cnt_b = (size_t)h.cnt_b; dist.nz = (size_t)h.nz;
  dist.C = h.C; dist.Sigma = h.Sigma;
  download(dist.vCl, h.vCl, (size_t)h.cnt_b);
  download(dist.vCs, h.vCs, (size_t)h.cnt_b);
  download(dist.vBs, h.vBs, (size_t)h.cnt_b);
  download(dist.vSBs, h.vSBs, (size_t)h.cnt_b);
  download(dist.vCol, h.vCol, (size_t)h.len);
  download(dist.vVal, h.vVal, (size_t)h.len);
  download(dist.vPerm, h.vPerm, (size_t)h.m);
  dist.vPartition.clear();
  M->sell = h;
  dist.rvvla_dev.set(hold.release());
}

int sell_call(const rvvla_sell* d, int stage, double a, const double* x, double b, double* y) {
  return rvvla_sell_spmv_f64(d, stage, a, x, b, y, nullptr);
}
int sell_call(const rvvla_sell* d, int stage, float a, const float* x, float b, float* y) {
  return rvvla_sell_spmv_f32(d, stage, a, x, b, y, nullptr);
}

// ------------------------------------------------------------------ CSR5
template <class T>
DeviceMirror& csr5_mirror(const spMtxCSR5<T>& A) {
  if (A.rvvla_dev.get()) return *A.rvvla_dev.get();
  DeviceMirror& M = fresh_mirror(A);
  rvvla_csr5& d = M.csr5;
  d.m = A._m; d.n = A._n; d.nnz = A._nnz;
  d.bit_y_offset = A._bit_y_offset; d.bit_seg_offset = A._bit_seg_offset; d.tile_desc_len = A._tile_desc_len;
  d.tail_tile_start = A._tail_tile_start; d.p = A._p; d.omega = A._omega; d.sigma = A._sigma;
  d.num_offsets = A._num_offsets;
  d.csr_row_pointer = upload(M, A._csr_row_pointer.data(), A._csr_row_pointer.size());
  d.csr_column_index = upload(M, A._csr_column_index.data(), A._csr_column_index.size());
  d.csr_value = upload(M, A._csr_value.data(), A._csr_value.size());
  d.tile_pointer = upload(M, A._csr5_tile_pointer.data(), A._csr5_tile_pointer.size());
  d.tile_descriptor = upload(M, A._csr5_tile_descriptor.data(), A._csr5_tile_descriptor.size());
  d.tile_empty_offset_pointer =
      upload(M, A._csr5_tile_empty_offset_pointer.data(), A._csr5_tile_empty_offset_pointer.size());
  d.tile_empty_offset = upload(M, A._csr5_tile_empty_offset.data(), A._csr5_tile_empty_offset.size());
  d.no_empty_rows = 0;  // always safe
  return M;
}

template <class T>
void csr5_build_from(spMtxCSR5<T>& dist, const rvvla_crs& src, const convertParams& p) {
  const int omega = param_i(p, "omega", 32);
  const int sigma = param_i(p, "sigma", 16);
  auto* M = new DeviceMirror();
  std::unique_ptr<DeviceMirror, void (*)(DeviceMirror*)> hold(M, rvvla_dropin::release);
  const int rc = rvvla_csr5_build(&src, val_bytes<T>(), omega, sigma, &M->co, nullptr);
  if (rc) throw_build(rc, "convert<spMtxCSR5>");
  const rvvla_csr5& h = M->co.h;
  dist._m = (int)h.m; dist._n = (int)h.n; dist._nnz = (int)h.nnz;
  dist._bit_y_offset = h.bit_y_offset; dist._bit_seg_offset = h.bit_seg_offset;
  dist._tile_desc_len = h.tile_desc_len; dist._tail_tile_start = h.tail_tile_start;
  dist._p = h.p; dist._omega = h.omega; dist._sigma = h.sigma; dist._num_offsets = h.num_offsets;
  const size_t nfull = h.p > 1 ? (size_t)(h.p - 1) : 0;
  download(dist._csr_row_pointer, h.csr_row_pointer, (size_t)h.m + 1);
  download(dist._csr_column_index, h.csr_column_index, (size_t)h.nnz);
  download(dist._csr_value, h.csr_value, (size_t)h.nnz);
  download(dist._csr5_tile_pointer, h.tile_pointer, (size_t)h.p + 1);
  download(dist._csr5_tile_descriptor, h.tile_descriptor, nfull * (size_t)h.omega * (size_t)h.tile_desc_len);
  download(dist._csr5_tile_empty_offset_pointer, h.tile_empty_offset_pointer, (size_t)h.p);
  download(dist._csr5_tile_empty_offset, h.tile_empty_offset, (size_t)h.num_offsets);
  dist._temp_calibrator.clear();
  dist.rvvla_set_format(CSR5_FORMAT_CSR5);
  M->csr5 = h;
  dist.rvvla_dev.set(hold.release());
}

int csr5_call(const rvvla_csr5* d, double a, const double* x, double b, double* y) {
  return rvvla_csr5_spmv_f64(d, a, x, b, y, nullptr);
}
int csr5_call(const rvvla_csr5* d, float a, const float* x, float b, float* y) {
  return rvvla_csr5_spmv_f32(d, a, x, b, y, nullptr);
}

// ------------------------------------------------------------------ LAV
template <class T>
DeviceMirror& lav_mirror(const spMtxLAV<T>& A) {
  if (A.rvvla_dev.get()) return *A.rvvla_dev.get();
  DeviceMirror& S = crs_mirror(A.sparse_part);  // the sparse part keeps its own mirror
  DeviceMirror& M = fresh_mirror(A);
  rvvla_lav& d = M.lav;
  d.SIMD_Lanes = (int64_t)A.SIMD_Lanes; d.m = A.m; d.n = A.n; d.nz = A.nz;
  d.segment_count = (int64_t)A.segment_count; d.chunk_count = (int64_t)A.chunk_count;
  d.segment_len = A.segment_len; d.n_steps = (int64_t)A.mask.size(); d.T = A.T;
  d.chunk_offsets = upload(M, A.chunk_offsets.data(), A.chunk_offsets.size());
  d.chunk_offsets_full_mask = upload(M, A.chunk_offsets_full_mask.data(), A.chunk_offsets_full_mask.size());
  std::vector<uint64_t> sp(A.segment_ptr.begin(), A.segment_ptr.end());
  d.segment_ptr = upload(M, sp.data(), sp.size());
  d.out_order = upload(M, A.out_order.data(), A.out_order.size());
  d.mask = upload(M, A.mask.data(), A.mask.size());
  d.val = upload(M, A.val.data(), A.val.size());
  d.col_id = upload(M, A.col_id.data(), A.col_id.size());
  d.sparse_part = S.crs;
  return M;
}

template <class T>
void lav_convert(spMtxLAV<T>& dist, const spMtxCRS<T>& src, const convertParams& p) {
  const int lanes = param_i(p, "SIMD_Lanes", 8);
  const double Tt = param_d(p, "T", 0.2);
  const int seglen = param_i(p, "segment_len", 40000);
  DeviceMirror& S = crs_mirror(src);
  rvvla_lav_owned o{};
  const int rc = rvvla_lav_build(&S.crs, val_bytes<T>(), lanes, Tt, seglen, &o, nullptr);
  if (rc) throw_build(rc, "convert<spMtxLAV>");
  try {
    const rvvla_lav& h = o.h;
    dist.SIMD_Lanes = (size_t)h.SIMD_Lanes; dist.m = (int)h.m; dist.n = (int)h.n; dist.nz = (int)h.nz;
    dist.segment_count = (size_t)h.segment_count; dist.chunk_count = (size_t)h.chunk_count;
    dist.T = h.T; dist.segment_len = (int)h.segment_len;
    const size_t L = (size_t)h.SIMD_Lanes, cc = (size_t)h.chunk_count, ns = (size_t)h.segment_count;
    download(dist.chunk_offsets, h.chunk_offsets, (cc + 1) * ns);
    download(dist.chunk_offsets_full_mask, h.chunk_offsets_full_mask, cc * ns);
    std::vector<uint64_t> sp;
    download(sp, h.segment_ptr, ns + 1);
    dist.segment_ptr.assign(sp.begin(), sp.end());
    download(dist.out_order, h.out_order, ns * cc * L);
    download(dist.mask, h.mask, (size_t)h.n_steps);
    download(dist.val, h.val, (size_t)h.n_steps * L);
    download(dist.col_id, h.col_id, (size_t)h.n_steps * L);
    const size_t snz = (size_t)h.sparse_part.nz;
    spMtxCRS<T> sp_part((size_t)h.m, (size_t)h.n, snz);
    if (h.m >= 0) check(rvvla_memcpy(sp_part.Rst, h.sparse_part.Rst, ((size_t)h.m + 1) * sizeof(int), nullptr), "rvvla_memcpy");
    if (snz) {
      check(rvvla_memcpy(sp_part.Col, h.sparse_part.Col, snz * sizeof(int), nullptr), "rvvla_memcpy");
      check(rvvla_memcpy(sp_part.Val, h.sparse_part.Val, snz * sizeof(T), nullptr), "rvvla_memcpy");
    }
    dist.sparse_part = std::move(sp_part);
  } catch (...) {
    rvvla_lav_free(&o);
    throw;
  }
  rvvla_lav_free(&o);  // the device copy is rebuilt from the host fields on first use
  dist.rvvla_dev.reset();
}

int lav_call(const rvvla_lav* d, double a, const double* x, double b, double* y) {
  return rvvla_lav_spmv_f64(d, a, x, b, y, nullptr);
}
int lav_call(const rvvla_lav* d, float a, const float* x, float b, float* y) {
  return rvvla_lav_spmv_f32(d, a, x, b, y, nullptr);
}

// ------------------------------------------------------------------ VHCC
template <class T>
DeviceMirror& vhcc_mirror(const spMtxVHCC<T>& A) {
  if (A.rvvla_dev.get()) return *A.rvvla_dev.get();
  DeviceMirror& M = fresh_mirror(A);
  rvvla_vhcc& d = M.vhcc;
  d.num_rows = (int64_t)A._num_rows; d.num_cols = (int64_t)A._num_cols; d.num_entries = (int64_t)A._num_entries;
  d.num_vectors = (int64_t)A._num_vectors; d.pad_entries = (int64_t)A._pad_entries; d.pad_rows = (int64_t)A._pad_rows;
  d.num_threads = (int32_t)A.params.num_threads; d.num_panels = (int32_t)A.params.num_panels;
  d.tile_row = (int32_t)A.params.tile_row; d.tile_col = (int32_t)A.params.tile_col;
  d.vec_size = (int32_t)A.params.vec_size; d.n_masks = (int32_t)A.params.n_masks;
  static_assert(sizeof(thr_info_t) == 10 * sizeof(int), "thr_info_t is 10 ints");
  d.thr_info = reinterpret_cast<const int32_t*>(upload(M, A._thr_info.data(), A._thr_info.size()));
  d.veceor_ptr = upload(M, A._veceor_ptr.data(), A._veceor_ptr.size());
  d.n_eor = (int64_t)A._veceor_ptr.size();
  d.scan_mask = upload(M, A._scan_mask.data(), A._scan_mask.size());
  d.scan_mask_bytes = (int64_t)A._scan_mask.size();
  d.row_arr = upload(M, A._row_arr.data(), A._row_arr.size());
  d.n_rowarr = (int64_t)A._row_arr.size();
  d.col_arr = upload(M, A._col_arr.data(), A._col_arr.size());
  d.vals_arr = upload(M, A._vals_arr.data(), A._vals_arr.size());
  return M;
}

template <class T>
void vhcc_convert(spMtxVHCC<T>& dist, const spMtxCRS<T>& src, const convertParams& p) {
  const int nt = param_i(p, "num_threads", 0);
  DeviceMirror& S = crs_mirror(src);
  auto* M = new DeviceMirror();
  std::unique_ptr<DeviceMirror, void (*)(DeviceMirror*)> hold(M, rvvla_dropin::release);
  const int rc = rvvla_vhcc_build(&S.crs, val_bytes<T>(), nt, &M->wo, nullptr);
  if (rc) throw_build(rc, "convert<spMtxVHCC>");
  const rvvla_vhcc& h = M->wo.h;
  dist.set_params(vhcc_params((size_t)h.num_threads, (size_t)h.num_panels, (size_t)h.tile_row, (size_t)h.tile_col,
                              (size_t)h.vec_size));
  dist.set_properties((size_t)h.num_rows, (size_t)h.num_cols, (size_t)h.num_entries, (size_t)h.num_vectors,
                      (size_t)h.pad_entries, (size_t)h.pad_rows);
  dist._nnz_per_panel = (size_t)h.num_entries;
  dist._extended_rows = (size_t)h.pad_rows;
  dist._thr_info.resize((size_t)h.num_threads);
  if (h.num_threads)
    check(rvvla_memcpy(dist._thr_info.data(), h.thr_info, (size_t)h.num_threads * sizeof(thr_info_t), nullptr),
          "rvvla_memcpy");
  download(dist._veceor_ptr, h.veceor_ptr, (size_t)h.n_eor);
  download(dist._scan_mask, h.scan_mask, (size_t)h.scan_mask_bytes);
  download(dist._row_arr, h.row_arr, (size_t)h.n_rowarr);
  download(dist._col_arr, h.col_arr, (size_t)(h.num_vectors * h.vec_size));
  download(dist._vals_arr, h.vals_arr, (size_t)(h.num_vectors * h.vec_size));
  M->vhcc = h;
  dist.rvvla_dev.set(hold.release());
}

int vhcc_call(const rvvla_vhcc* d, double a, const double* x, double b, double* y) {
  return rvvla_vhcc_spmv_f64(d, a, x, b, y, nullptr);
}
int vhcc_call(const rvvla_vhcc* d, float a, const float* x, float b, float* y) {
  return rvvla_vhcc_spmv_f32(d, a, x, b, y, nullptr);
}

// ------------------------------------------------------------------ CVR
template <class T>
DeviceMirror& cvr_mirror(const spMtxCVR<T>& A) {
  if (A.rvvla_dev.get()) return *A.rvvla_dev.get();
  DeviceMirror& M = fresh_mirror(A);
  rvvla_cvr& d = M.cvr;
  d.nItems = (int64_t)A.nItems; d.numRows = (int64_t)A.numRows; d.numCols = (int64_t)A.numCols;
  d.SIMD_LEN = (int32_t)A.SIMD_LEN; d.Nthreads = A.Nthreads; d.Nthreads_avail = A.Nthreads_avail;
  d.no_empty_rows = 0;
  d.vPack_vec_vals = upload(M, A.vPack_vec_vals.data(), A.vPack_vec_vals.size());
  d.vPack_vec_cols = upload(M, A.vPack_vec_cols.data(), A.vPack_vec_cols.size());
  d.vPack_vec_record = upload(M, A.vPack_vec_record.data(), A.vPack_vec_record.size());
  d.n_record = (int64_t)A.vPack_vec_record.size();
  d.writeback_pos_record = upload(M, A.writeback_pos_record.data(), A.writeback_pos_record.size());
  d.n_writeback = (int64_t)A.writeback_pos_record.size();
  return M;
}

template <class T>
void cvr_convert(spMtxCVR<T>& dist, const spMtxCRS<T>& src, const convertParams& p) {
  const int nt = param_i(p, "Nthreads", 0);
  DeviceMirror& S = crs_mirror(src);
  auto* M = new DeviceMirror();
  std::unique_ptr<DeviceMirror, void (*)(DeviceMirror*)> hold(M, rvvla_dropin::release);
  const int rc = rvvla_cvr_build(&S.crs, val_bytes<T>(), nt, &M->ro, nullptr);
  if (rc) throw_build(rc, "convert<spMtxCVR>");
  const rvvla_cvr& h = M->ro.h;
  dist.nItems = (size_t)h.nItems; dist.numRows = (size_t)h.numRows; dist.numCols = (size_t)h.numCols;
  dist.SIMD_LEN = (size_t)h.SIMD_LEN; dist.Nthreads = h.Nthreads; dist.Nthreads_avail = h.Nthreads_avail;
  download(dist.vPack_vec_vals, h.vPack_vec_vals, (size_t)h.nItems);
  download(dist.vPack_vec_cols, h.vPack_vec_cols, (size_t)h.nItems);
  download(dist.vPack_vec_record, h.vPack_vec_record, (size_t)h.n_record);
  download(dist.writeback_pos_record, h.writeback_pos_record, (size_t)h.n_writeback);
  M->cvr = h;
  dist.rvvla_dev.set(hold.release());
}

int cvr_call(const rvvla_cvr* d, double a, const double* x, double b, double* y) {
  return rvvla_cvr_spmv_f64(d, a, x, b, y, nullptr);
}
int cvr_call(const rvvla_cvr* d, float a, const float* x, float b, float* y) {
  return rvvla_cvr_spmv_f32(d, a, x, b, y, nullptr);
}

// ------------------------------------------------------------------ VNEC
int vnec_call(const rvvla_vnec* d, double a, const double* x, double b, double* y) {
  return rvvla_vnec_spmv_f64(d, a, x, b, y, nullptr);
}
int vnec_call(const rvvla_vnec* d, float a, const float* x, float b, float* y) {
  return rvvla_vnec_spmv_f32(d, a, x, b, y, nullptr);
}

template <class T>
sparse_matrix_status unsupported_op() {
  sparse_matrix_status st;
  st.code = RVVLA_ERR_UNSUPPORTED;
  return st;
}

}  // namespace

// ------------------------------------------------------------------ VNEC init
template <class V>
void rvvla_vnec_init(spMtxVNEC<V>& A, int nthreads) {
  if (!A.G) return;
  DeviceMirror& S = crs_mirror(*A.G);
  auto* M = new DeviceMirror();
  std::unique_ptr<DeviceMirror, void (*)(DeviceMirror*)> hold(M, rvvla_dropin::release);
  const int rc = rvvla_vnec_build(&S.crs, (int)sizeof(V), nthreads, -1, &M->vo, nullptr);
  if (rc) throw_build(rc, "spMtxVNEC");
  const rvvla_vnec& h = M->vo.h;
  A.NUM_THREADS_VNEC = h.NUM_THREADS_VNEC;
  A.IRD_mat = h.IRD_mat;
  A.vnec_t = (SpB_VNEC_type)h.vnec_t;
  A.num_merge_items = (int)(h.nz + h.m);
  A.items_per_thread = (A.num_merge_items + A.NUM_THREADS_VNEC - 1) / std::max(A.NUM_THREADS_VNEC, 1);
  M->vnec = h;
  A.rvvla_dev.set(hold.release());
}
template void rvvla_vnec_init<double>(spMtxVNEC<double>&, int);
template void rvvla_vnec_init<float>(spMtxVNEC<float>&, int);

// ------------------------------------------------------------------ CSR5 members
template <class ValT>
int spMtxCSR5<ValT>::inputCSR(int m, int n, int nnz, int* rp, int* ci, ValT* v) {
  freeMem();
  _m = m;
  _n = n;
  _nnz = nnz;
  _csr_row_pointer.assign(rp, rp + m + 1);
  _csr_column_index.assign(reinterpret_cast<uint32_t*>(ci), reinterpret_cast<uint32_t*>(ci) + nnz);
  _csr_value.assign(v, v + nnz);
  _format = CSR5_FORMAT_CSR;
  return CSR5_SUCCESS;
}

template <class ValT>
int spMtxCSR5<ValT>::asCSR5(const convertParams& params) {
  if (_format == CSR5_FORMAT_CSR5) return CSR5_SUCCESS;
  if (_format != CSR5_FORMAT_CSR) return CSR5_UNKNOWN_FORMAT;
  if (param_i(params, "omega", 32) != 32) return CSR5_UNSUPPORTED_OMEGA;
  try {
    spMtxCRS<ValT> crs((size_t)_m, (size_t)_n, (size_t)_nnz, _csr_row_pointer.data(),
                       reinterpret_cast<const int*>(_csr_column_index.data()), _csr_value.data());
    DeviceMirror& S = crs_mirror(crs);
    csr5_build_from(*this, S.crs, params);
  } catch (...) {
    return CSR5_CONVERTION_FAILED;
  }
  _format = CSR5_FORMAT_CSR5;
  return CSR5_SUCCESS;
}

template class spMtxCSR5<double>;
template class spMtxCSR5<float>;

// ------------------------------------------------------------------ overloads
#define RVVLA_DROPIN_SPMV(CLS, T, BODY)                                                                     \
  sparse_matrix_status rvvla_sparse_mv(sparse_operation_t op, T alpha, const CLS<T>& A,                      \
                                       const std::vector<T>& b, T beta, std::vector<T>& y,                   \
                                       sparse_matrix_mv_stage stage) {                                       \
    BODY                                                                                                      \
  }

#define RVVLA_DROPIN_SIMPLE(CLS, T, MIRROR, FIELD, CALL, ROWS, COLS)                                         \
  RVVLA_DROPIN_SPMV(CLS, T, {                                                                                 \
    if (op != SPARSE_OPERATION_NON_TRANSPOSE) return unsupported_op<T>();                                    \
    return guarded([&] {                                                                                     \
      if (!multiplies(stage)) return sparse_matrix_status{};                                                 \
      DeviceMirror& M = MIRROR(A);                                                                            \
      return run<T>(M, (size_t)(ROWS), (size_t)(COLS), b, beta, y, false,                                    \
                    [&](const T* x, T* yy) { return CALL(&M.FIELD, alpha, x, beta, yy); });                  \
    });                                                                                                       \
  })

RVVLA_DROPIN_SPMV(spMtxCRS, double, { return crs_spmv<double>(op, alpha, A, b, beta, y, stage); })
RVVLA_DROPIN_SPMV(spMtxCRS, float, { return crs_spmv<float>(op, alpha, A, b, beta, y, stage); })
RVVLA_DROPIN_SIMPLE(spMtxHCSR, double, hcsr_mirror, hcsr, hcsr_call, A.m, A.n)
RVVLA_DROPIN_SIMPLE(spMtxHCSR, float, hcsr_mirror, hcsr, hcsr_call, A.m, A.n)

// CSR5 products need the tile layout: an object holding only the CSR input
// (inputCSR without asCSR5) is rejected with RVVLA_ERR_FORMAT.
template <class T>
sparse_matrix_status csr5_spmv(sparse_operation_t op, T alpha, const spMtxCSR5<T>& A, const std::vector<T>& b,
                               T beta, std::vector<T>& y, sparse_matrix_mv_stage stage) {
  if (op != SPARSE_OPERATION_NON_TRANSPOSE) return unsupported_op<T>();
  if (A.format() != CSR5_FORMAT_CSR5) {
    sparse_matrix_status st;
    st.code = RVVLA_ERR_FORMAT;
    return st;
  }
  return guarded([&] {
    if (!multiplies(stage)) return sparse_matrix_status{};
    DeviceMirror& M = csr5_mirror(A);
    return run<T>(M, (size_t)A._m, (size_t)A._n, b, beta, y, false,
                  [&](const T* x, T* yy) { return csr5_call(&M.csr5, alpha, x, beta, yy); });
  });
}
RVVLA_DROPIN_SPMV(spMtxCSR5, double, { return csr5_spmv<double>(op, alpha, A, b, beta, y, stage); })
RVVLA_DROPIN_SPMV(spMtxCSR5, float, { return csr5_spmv<float>(op, alpha, A, b, beta, y, stage); })
RVVLA_DROPIN_SIMPLE(spMtxLAV, double, lav_mirror, lav, lav_call, A.m, A.n)
RVVLA_DROPIN_SIMPLE(spMtxLAV, float, lav_mirror, lav, lav_call, A.m, A.n)
RVVLA_DROPIN_SIMPLE(spMtxVHCC, double, vhcc_mirror, vhcc, vhcc_call, A._num_rows, A._num_cols)
RVVLA_DROPIN_SIMPLE(spMtxVHCC, float, vhcc_mirror, vhcc, vhcc_call, A._num_rows, A._num_cols)
RVVLA_DROPIN_SIMPLE(spMtxCVR, double, cvr_mirror, cvr, cvr_call, A.numRows, A.numCols)
RVVLA_DROPIN_SIMPLE(spMtxCVR, float, cvr_mirror, cvr, cvr_call, A.numRows, A.numCols)

template <class T>
sparse_matrix_status vnec_spmv(sparse_operation_t op, T alpha, const spMtxVNEC<T>& A, const std::vector<T>& b,
                               T beta, std::vector<T>& y, sparse_matrix_mv_stage stage) {
  if (op != SPARSE_OPERATION_NON_TRANSPOSE) return unsupported_op<T>();
  return guarded([&] {
    if (!multiplies(stage)) return sparse_matrix_status{};
    if (!A.rvvla_dev.get()) {
      if (!A.G) {
        sparse_matrix_status st;
        st.code = RVVLA_ERR_INVALID_ARG;
        return st;
      }
      rvvla_vnec_init(const_cast<spMtxVNEC<T>&>(A), A.NUM_THREADS_VNEC);
    }
    DeviceMirror& M = *A.rvvla_dev.get();
    return run<T>(M, (size_t)M.vnec.m, (size_t)M.vnec.n, b, beta, y, false,
                  [&](const T* x, T* yy) { return vnec_call(&M.vnec, alpha, x, beta, yy); });
  });
}
RVVLA_DROPIN_SPMV(spMtxVNEC, double, { return vnec_spmv<double>(op, alpha, A, b, beta, y, stage); })
RVVLA_DROPIN_SPMV(spMtxVNEC, float, { return vnec_spmv<float>(op, alpha, A, b, beta, y, stage); })

// SELL-C-sigma: the stages act on y (PREPARATION permutes it into the sorted
// row order, GET_RESULTS restores it), so y is staged for every stage but
// ALL_STAGES with beta == 0.
template <class T>
sparse_matrix_status sell_spmv(sparse_operation_t op, T alpha, const spMtxSELL_C_Sigma<T>& A,
                               const std::vector<T>& b, T beta, std::vector<T>& y, sparse_matrix_mv_stage stage) {
  if (op != SPARSE_OPERATION_NON_TRANSPOSE) return unsupported_op<T>();
  return guarded([&] {
    DeviceMirror& M = sell_mirror(A);
    const bool reads_y = stage != SPARSE_MATRIX_MV_ALL_STAGES;
    return run<T>(M, A.m, A.n, b, beta, y, reads_y,
                  [&](const T* x, T* yy) { return sell_call(&M.sell, (int)stage, alpha, x, beta, yy); });
  });
}
RVVLA_DROPIN_SPMV(spMtxSELL_C_Sigma, double, { return sell_spmv<double>(op, alpha, A, b, beta, y, stage); })
RVVLA_DROPIN_SPMV(spMtxSELL_C_Sigma, float, { return sell_spmv<float>(op, alpha, A, b, beta, y, stage); })

// ------------------------------------------------------------------ mixed precision
#define RVVLA_DROPIN_MIXED(CLS, MIRROR, FIELD, FN, ROWS, COLS)                                                \
  sparse_matrix_status rvvla_sparse_mv_mixed(sparse_operation_t op, float alpha, const CLS<float>& A,          \
                                             const std::vector<float>& b, float beta, std::vector<float>& y) { \
    if (op != SPARSE_OPERATION_NON_TRANSPOSE) return unsupported_op<float>();                                 \
    return guarded([&] {                                                                                       \
      DeviceMirror& M = MIRROR(A);                                                                             \
      return run<float>(M, (size_t)(ROWS), (size_t)(COLS), b, beta, y, false, [&](const float* x, float* yy) { \
        return FN(&M.FIELD, RVVLA_F32, alpha, x, beta, yy, nullptr);                                           \
      });                                                                                                      \
    });                                                                                                        \
  }

RVVLA_DROPIN_MIXED(spMtxCRS, crs_mirror, crs, rvvla_crs_spmv_mixed, A.m, A.n)
RVVLA_DROPIN_MIXED(spMtxHCSR, hcsr_mirror, hcsr, rvvla_hcsr_spmv_mixed, A.m, A.n)
RVVLA_DROPIN_MIXED(spMtxSELL_C_Sigma, sell_mirror, sell, rvvla_sell_spmv_mixed, A.m, A.n)

sparse_matrix_status rvvla_sparse_mv_mixed(sparse_operation_t op, float alpha, const spMtxCSR5<float>& A,
                                           const std::vector<float>& b, float beta, std::vector<float>& y) {
  if (op != SPARSE_OPERATION_NON_TRANSPOSE) return unsupported_op<float>();
  if (A.format() != CSR5_FORMAT_CSR5) {
    sparse_matrix_status st;
    st.code = RVVLA_ERR_FORMAT;
    return st;
  }
  return guarded([&] {
    DeviceMirror& M = csr5_mirror(A);
    return run<float>(M, (size_t)A._m, (size_t)A._n, b, beta, y, false, [&](const float* x, float* yy) {
      return rvvla_csr5_spmv_mixed(&M.csr5, RVVLA_F32, alpha, x, beta, yy, nullptr);
    });
  });
}

#define RVVLA_DROPIN_CONVERT(CLS, FN)                                                                        \
  void rvvla_convert(CLS<double>& dist, const spMtxCRS<double>& src, const convertParams& p) { FN(dist, src, p); } \
  void rvvla_convert(CLS<float>& dist, const spMtxCRS<float>& src, const convertParams& p) { FN(dist, src, p); }

template <class T>
void csr5_convert(spMtxCSR5<T>& dist, const spMtxCRS<T>& src, const convertParams& p) {
  if (param_i(p, "omega", 32) != 32) throw std::invalid_argument("convert<spMtxCSR5>: omega must be 32 on the GPU");
  DeviceMirror& S = crs_mirror(src);
  csr5_build_from(dist, S.crs, p);
}

RVVLA_DROPIN_CONVERT(spMtxHCSR, hcsr_convert)
RVVLA_DROPIN_CONVERT(spMtxSELL_C_Sigma, sell_convert)
RVVLA_DROPIN_CONVERT(spMtxCSR5, csr5_convert)
RVVLA_DROPIN_CONVERT(spMtxLAV, lav_convert)
RVVLA_DROPIN_CONVERT(spMtxVHCC, vhcc_convert)
RVVLA_DROPIN_CONVERT(spMtxCVR, cvr_convert)

// ------------------------------------------------------------------ autotuner
namespace {

template <class T>
convertParams tune(int fmt, const spMtxCRS<T>& src, bool mixed, int iters) {
  DeviceMirror& S = crs_mirror(src);
  rvvla_tune_params best{};
  double ms = 0.0;
  const int vt = std::is_same<T, double>::value ? RVVLA_F64 : RVVLA_F32;
  const int rc = rvvla_autotune(fmt, &S.crs, vt, mixed ? 1 : 0, iters, &best, &ms, nullptr, nullptr, 0, nullptr,
                                nullptr);
  if (rc) throw_build(rc, "autotune");
  convertParams p;
  switch (fmt) {
    case RVVLA_FMT_HCSR:
      p.param["R"].i = (int)best.R;
      p.param["C"].i = (int)best.C;
      p.param["p"].d = best.p;
      break;
    case RVVLA_FMT_SELL:
      p.param["C"].i = (int)best.C;
      p.param["Sigma"].i = (int)best.sigma;
      break;
    case RVVLA_FMT_CSR5:
      p.param["omega"].i = 32;
      p.param["sigma"].i = (int)best.sigma;
      break;
    case RVVLA_FMT_LAV:
      p.param["SIMD_Lanes"].i = (int)best.simd_lanes;
      p.param["T"].d = best.T;
      p.param["segment_len"].i = (int)best.segment_len;
      break;
    case RVVLA_FMT_VHCC:
      p.param["num_threads"].i = (int)best.threads;
      break;
    default:
      p.param["Nthreads"].i = (int)best.threads;
      break;
  }
  return p;
}

}  // namespace

#define RVVLA_DROPIN_TUNE(CLS, FMT)                                                                          \
  convertParams rvvla_autotune_for(const CLS<double>*, const spMtxCRS<double>& src, bool mixed, int iters) { \
    return tune<double>(FMT, src, mixed, iters);                                                              \
  }                                                                                                           \
  convertParams rvvla_autotune_for(const CLS<float>*, const spMtxCRS<float>& src, bool mixed, int iters) {   \
    return tune<float>(FMT, src, mixed, iters);                                                               \
  }

RVVLA_DROPIN_TUNE(spMtxHCSR, RVVLA_FMT_HCSR)
RVVLA_DROPIN_TUNE(spMtxSELL_C_Sigma, RVVLA_FMT_SELL)
RVVLA_DROPIN_TUNE(spMtxCSR5, RVVLA_FMT_CSR5)
RVVLA_DROPIN_TUNE(spMtxLAV, RVVLA_FMT_LAV)
RVVLA_DROPIN_TUNE(spMtxVHCC, RVVLA_FMT_VHCC)
RVVLA_DROPIN_TUNE(spMtxCVR, RVVLA_FMT_CVR)

}  // namespace SparseMatrixLib
