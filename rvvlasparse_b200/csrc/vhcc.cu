// vhcc.cu — spMtxVHCC on sm_100a: GPU builder (vec_size 32) and SpMV.
//
// Layout (include/VHCC.h:43-112 of the reference; kernel
// src/rvv/spmv_vhcc.cpp:73-162 fp64, :164-250 fp32): nonzeros in CSR order
// packed into vectors of vec_size lanes (zero padded); VHCC threads own
// vector ranges; vectors holding a "write lane" (a row's last nonzero, or a
// thread range's last lane, written to the thread's overflow row
// num_rows + tid) are listed in veceor_ptr (per thread, then a sentinel) with
// n_masks scan masks and one write mask each; row_arr lists the write lanes'
// rows; thr_info[tid] = {vbase, rbase, sbase (bytes), last_row,
// overflow_row, start_vec, end_vec, panel_id, merge_start, merge_end}.  The
// reference ships no builder (VHCC.h:80-112 holds setters for one); this one
// matches the oracle's builder bit for bit at vec_size 32.
//
// SpMV: one warp per VHCC thread, lane = vector lane.  Lanes accumulate
// their products; at an end-of-row vector the warp runs the reference's
// masked slide-up scan as five __shfl_up steps gated by the stored masks,
// stores the write lanes' sums to tmp[row_arr[...]] and carries lane 31 into
// the next vector (:104-140).  Overflow rows are merged into last_row in
// thread order by a second kernel (the reference's atomic, :157-161), and a
// third computes y = alpha*tmp + beta*y (:335-397).  Deterministic.
#include <algorithm>
#include <cstring>
#include <string>

#include "crs_merge.cuh"
#include "rvvla_internal.cuh"
#include "scan.cuh"

namespace rvvla {
namespace {

constexpr int kVec = 32;
constexpr int kMasks = 5;  // log2(32)
constexpr int kVhccU = 4;  // vectors whose loads are in flight together

// ---------------------------------------------------------------- builder
__global__ void vhcc_mark_kernel(int64_t m, const int* __restrict__ Rst, uint32_t* __restrict__ endbits,
                                 int* __restrict__ endrow) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= m) return;
  const int a = Rst[r], b = Rst[r + 1];
  if (b > a) {
    atomicOr(&endbits[(b - 1) / kVec], 1u << ((b - 1) % kVec));
    endrow[b - 1] = (int)r;
  }
}

__device__ __forceinline__ int64_t vhcc_v0(int64_t nvec, int64_t NT, int64_t t) { return nvec * t / NT; }

// pass 1: per VHCC thread, count end-of-row vectors and write lanes
__global__ void vhcc_count_kernel(int64_t nvec, int64_t NT, const uint32_t* __restrict__ endbits,
                                  int64_t* __restrict__ neor, int64_t* __restrict__ nrows) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= NT) return;
  const int64_t v0 = vhcc_v0(nvec, NT, t), v1 = vhcc_v0(nvec, NT, t + 1);
  int64_t e = 0, r = 0;
  for (int64_t v = v0; v < v1; ++v) {
    uint32_t w = endbits[v];
    if (v == v1 - 1) w |= 1u << (kVec - 1);
    if (w) { e++; r += __popc(w); }
  }
  neor[t] = e;
  nrows[t] = r;
}

// pass 2: veceor_ptr, scan masks, row_arr, thr_info
__global__ void vhcc_fill_kernel(int64_t nvec, int64_t NT, int64_t m, int64_t nnz, const int* __restrict__ Rst,
                                 const uint32_t* __restrict__ endbits, const int* __restrict__ endrow,
                                 const int64_t* __restrict__ eorofs, const int64_t* __restrict__ rowofs,
                                 uint32_t* __restrict__ veceor, uint32_t* __restrict__ smask,
                                 uint32_t* __restrict__ row_arr, int* __restrict__ thr) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= NT) return;
  const int64_t v0 = vhcc_v0(nvec, NT, t), v1 = vhcc_v0(nvec, NT, t + 1);
  int64_t e = eorofs[t], r = rowofs[t];
  int* ti = thr + t * 10;
  ti[0] = (int)e;
  ti[1] = (int)r;
  ti[2] = (int)(e * (kMasks + 1) * (kVec / 8));
  ti[3] = (int)(m + t);
  ti[4] = (int)(m + t);
  ti[5] = (int)v0;
  ti[6] = (int)v1;
  ti[7] = ti[8] = ti[9] = 0;
  for (int64_t v = v0; v < v1; ++v) {
    const uint32_t real = endbits[v];
    const bool tend = (v == v1 - 1);
    const uint32_t w = real | (tend ? (1u << (kVec - 1)) : 0u);
    if (!w) continue;
    veceor[e] = (uint32_t)v;
    uint32_t* mk = smask + e * (kMasks + 1);
    for (int s = 0; s < kMasks; ++s) {
      const int d = 1 << s;
      uint32_t bits = 0;
      for (int i = d; i < kVec; ++i)
        if (((w >> (i - d)) & ((1u << d) - 1u)) == 0u) bits |= 1u << i;
      mk[s] = bits;
    }
    mk[kMasks] = w;
    for (int l = 0; l < kVec; ++l) {
      if (!((w >> l) & 1u)) continue;
      const int64_t k = v * kVec + l;
      if (tend && l == kVec - 1 && !((real >> l) & 1u)) {
        row_arr[r++] = (uint32_t)(m + t);
        int64_t last;
        if (k < nnz) {  // row of element k: largest q with Rst[q] <= k
          int64_t lo = 0, hi = m + 1;
          while (hi - lo > 1) {
            const int64_t mid = (lo + hi) >> 1;
            if (Rst[mid] <= k) lo = mid;
            else hi = mid;
          }
          last = lo;
        } else {
          int64_t lo = 0, hi = m + 1;
          const int64_t kk = nnz > 0 ? nnz - 1 : 0;
          while (hi - lo > 1) {
            const int64_t mid = (lo + hi) >> 1;
            if (Rst[mid] <= kk) lo = mid;
            else hi = mid;
          }
          last = nnz > 0 ? lo : 0;
        }
        ti[3] = (int)last;
      } else {
        row_arr[r++] = (uint32_t)endrow[k];
      }
    }
    e++;
  }
}

template <int VB>
__global__ void vhcc_pack_kernel(int64_t total, int64_t nnz, const int* __restrict__ Col, const uint8_t* __restrict__ Val,
                                 uint32_t* __restrict__ col, uint8_t* __restrict__ val) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= total) return;
  const bool in = k < nnz;
  col[k] = in ? (uint32_t)Col[k] : 0u;
#pragma unroll
  for (int q = 0; q < VB; ++q) val[k * VB + q] = in ? Val[k * VB + q] : 0;
}

// ---------------------------------------------------------------- SpMV
template <class V, class X, class Ac, class CT>
__global__ void __launch_bounds__(256)
vhcc_spmv_kernel(int64_t NT, const int* __restrict__ thr, const uint32_t* __restrict__ veceor,
                 const uint32_t* __restrict__ smask, const uint32_t* __restrict__ row_arr,
                 const uint32_t* __restrict__ col, const V* __restrict__ vals, const X* __restrict__ x,
                 CT* __restrict__ tmp) {
  const int64_t t = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (t >= NT) return;
  const int* ti = thr + t * 10;
  int64_t vidx = ti[0], ridx = ti[1];
  const uint32_t* mk = smask + ((int64_t)ti[2] >> 2);  // sbase is in bytes
  const int64_t v0 = ti[5], v1 = ti[6];
  uint32_t eor = veceor[vidx++];
  const uint64_t pf = policy_evict_first(), pl = policy_evict_last();
  CT res = 0;
  bool pending = false;  // vectors without a row end left partial sums in every lane
  // vectors kVhccU at a time: all their loads are issued first (indices past
  // the range clamped to its last vector, their products dropped)
  for (int64_t vb = v0; vb < v1; vb += kVhccU) {
    uint32_t cc[kVhccU];
    V av[kVhccU];
    X xv[kVhccU];
#pragma unroll
    for (int u = 0; u < kVhccU; ++u) cc[u] = ld_stream(col + min(vb + u, v1 - 1) * kVec + lane, pf);
#pragma unroll
    for (int u = 0; u < kVhccU; ++u) av[u] = ld_stream(vals + min(vb + u, v1 - 1) * kVec + lane, pf);
#pragma unroll
    for (int u = 0; u < kVhccU; ++u) xv[u] = ld_keep(x + cc[u], pl);
#pragma unroll
    for (int u = 0; u < kVhccU; ++u) {
      const int64_t v = vb + u;
      if (v >= v1) break;
      const CT prod = (CT)vmul(av[u], xv[u]);
      if ((uint32_t)v != eor) {
        res += prod;
        pending = true;
      } else {
        // all of those sums belong to the row that opens this vector: fold
        // them into lane 0 (the reference sums each such vector into its
        // first slot) before the segmented scan
        if (pending) {
#pragma unroll
          for (int off = 16; off > 0; off >>= 1) res += __shfl_xor_sync(0xffffffffu, res, off);
          res = (lane == 0) ? res : CT(0);
          pending = false;
        }
        res += prod;
#pragma unroll
        for (int s = 0; s < kMasks; ++s) {
          const CT o = __shfl_up_sync(0xffffffffu, res, 1 << s);
          if ((mk[s] >> lane) & 1u) res += o;
        }
        const uint32_t wm = mk[kMasks];
        if ((wm >> lane) & 1u) {
          const int rank = __popc(wm & ((1u << lane) - 1u));
          tmp[row_arr[ridx + rank]] = res;
        }
        ridx += __popc(wm);
        const CT carry = ((wm >> 31) & 1u) ? CT(0) : __shfl_sync(0xffffffffu, res, 31);
        res = (lane == 0) ? carry : CT(0);
        mk += kMasks + 1;
        eor = veceor[vidx++];
      }
    }
  }
}

// overflow rows into last_row, in thread order (the reference's atomic add)
template <class CT>
__global__ void vhcc_overflow_kernel(int64_t NT, int64_t m, const int* __restrict__ thr, CT* __restrict__ tmp) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= NT) return;
  const int r = thr[t * 10 + 3];
  if (r >= m) return;
  if (t > 0 && thr[(t - 1) * 10 + 3] == r) return;
  CT s = tmp[thr[t * 10 + 4]];
  for (int64_t u = t + 1; u < NT && thr[u * 10 + 3] == r; ++u) s += tmp[thr[u * 10 + 4]];
  tmp[r] += s;
}

template <class X, class CT>
__global__ void vhcc_out_kernel(int64_t m, const CT* __restrict__ tmp, X* __restrict__ y, X alpha, X beta) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) write_row(y, (int)i, alpha, beta, (X)tmp[i]);
}

int vhcc_validate(const rvvla_vhcc* A, const void* x, const void* y) {
  if (!A) return fail(RVVLA_ERR_INVALID_ARG, "vhcc: null descriptor");
  if (A->num_rows < 0 || A->num_threads <= 0 || A->pad_rows < A->num_rows) return fail(RVVLA_ERR_INVALID_ARG, "vhcc: bad sizes");
  if (A->vec_size != kVec || A->n_masks != kMasks)
    return fail(RVVLA_ERR_UNSUPPORTED, "vhcc: the sm_100a kernel needs vec_size 32 (one vector lane per warp lane)");
  if (A->num_panels != 1) return fail(RVVLA_ERR_UNSUPPORTED, "vhcc: only one panel (as the reference's kernel)");
  if (A->num_rows > 0 && (!A->thr_info || !A->veceor_ptr || !A->scan_mask || !A->row_arr || !y))
    return fail(RVVLA_ERR_INVALID_ARG, "vhcc: null array");
  if (A->num_vectors > 0 && (!A->col_arr || !A->vals_arr || !x)) return fail(RVVLA_ERR_INVALID_ARG, "vhcc: null array");
  return RVVLA_OK;
}

template <class V, class X, class Ac, class CT>
int vhcc_spmv_impl(const rvvla_vhcc* A, X alpha, const X* x, X beta, X* y, cudaStream_t st) {
  int rc = vhcc_validate(A, x, y);
  if (rc) return rc;
  if (A->num_rows == 0) return RVVLA_OK;
  Scratch sc;
  RVVLA_CUDA(sc.alloc((size_t)A->pad_rows * sizeof(CT), st));
  CT* tmp = sc.as<CT>();
  RVVLA_CUDA(cudaMemsetAsync(tmp, 0, (size_t)A->pad_rows * sizeof(CT), st));
  const int64_t NT = A->num_threads;
  vhcc_spmv_kernel<V, X, Ac, CT><<<(unsigned)((NT * 32 + 255) / 256), 256, 0, st>>>(
      NT, A->thr_info, A->veceor_ptr, (const uint32_t*)A->scan_mask, A->row_arr, A->col_arr, (const V*)A->vals_arr, x,
      tmp);
  RVVLA_LAUNCHED("vhcc_spmv_kernel");
  vhcc_overflow_kernel<CT><<<(unsigned)((NT + 255) / 256), 256, 0, st>>>(NT, A->num_rows, A->thr_info, tmp);
  RVVLA_LAUNCHED("vhcc_overflow_kernel");
  vhcc_out_kernel<X, CT><<<(unsigned)((A->num_rows + 255) / 256), 256, 0, st>>>(A->num_rows, tmp, y, alpha, beta);
  RVVLA_LAUNCHED("vhcc_out_kernel");
  return RVVLA_OK;
}

int vhcc_build_impl(const rvvla_crs* src, int vb, int64_t NT, rvvla_vhcc_owned* out, cudaStream_t st) {
  if (!src || !out) return fail(RVVLA_ERR_INVALID_ARG, "vhcc_build: null argument");
  std::memset(out, 0, sizeof(*out));
  if (vb != 8 && vb != 4 && vb != 2) return fail(RVVLA_ERR_INVALID_ARG, "vhcc_build: val_bytes must be 8, 4 or 2");
  const int64_t m = src->m, nnz = src->nz;
  if (m < 0 || nnz < 0 || src->n < 0) return fail(RVVLA_ERR_INVALID_ARG, "vhcc_build: bad sizes");
  const int64_t nvec = (nnz + kVec - 1) / kVec;
  if (NT <= 0) NT = std::max<int64_t>(1, (nvec + 63) / 64);
  if (m + NT >= INT32_MAX || nnz >= INT32_MAX) return fail(RVVLA_ERR_TOO_LARGE, "vhcc_build: sizes beyond int32");
  rvvla_vhcc& h = out->h;
  h.num_rows = m; h.num_cols = src->n; h.num_entries = nnz; h.num_vectors = nvec;
  h.pad_entries = nvec * kVec - nnz; h.pad_rows = m + NT;
  h.num_threads = (int32_t)NT; h.num_panels = 1; h.tile_row = 512; h.tile_col = 512; h.vec_size = kVec;
  h.n_masks = kMasks;
  Scratch s_bits, s_erow, s_ne, s_nr, s_eo, s_ro;
  RVVLA_CUDA(s_bits.alloc((size_t)std::max<int64_t>(nvec, 1) * 4, st));
  RVVLA_CUDA(s_erow.alloc((size_t)std::max<int64_t>(nvec * kVec, 1) * 4, st));
  RVVLA_CUDA(s_ne.alloc((size_t)(NT + 1) * 8, st));
  RVVLA_CUDA(s_nr.alloc((size_t)(NT + 1) * 8, st));
  RVVLA_CUDA(s_eo.alloc((size_t)(NT + 1) * 8, st));
  RVVLA_CUDA(s_ro.alloc((size_t)(NT + 1) * 8, st));
  RVVLA_CUDA(cudaMemsetAsync(s_bits.p, 0, (size_t)std::max<int64_t>(nvec, 1) * 4, st));
  if (m > 0) {
    vhcc_mark_kernel<<<(unsigned)((m + 255) / 256), 256, 0, st>>>(m, src->Rst, s_bits.as<uint32_t>(), s_erow.as<int>());
    RVVLA_LAUNCHED("vhcc_mark_kernel");
  }
  vhcc_count_kernel<<<(unsigned)((NT + 255) / 256), 256, 0, st>>>(nvec, NT, s_bits.as<uint32_t>(), s_ne.as<int64_t>(),
                                                                   s_nr.as<int64_t>());
  RVVLA_LAUNCHED("vhcc_count_kernel");
  int rc = exclusive_scan_i64(s_ne.as<int64_t>(), s_eo.as<int64_t>(), NT, st);
  if (rc) return rc;
  rc = exclusive_scan_i64(s_nr.as<int64_t>(), s_ro.as<int64_t>(), NT, st);
  if (rc) return rc;
  int64_t n_eor = 0, n_rows = 0;
  RVVLA_CUDA(cudaMemcpyAsync(&n_eor, s_eo.as<int64_t>() + NT, 8, cudaMemcpyDeviceToHost, st));
  RVVLA_CUDA(cudaMemcpyAsync(&n_rows, s_ro.as<int64_t>() + NT, 8, cudaMemcpyDeviceToHost, st));
  RVVLA_CUDA(cudaStreamSynchronize(st));
  h.n_eor = n_eor + 1;
  h.scan_mask_bytes = n_eor * (kMasks + 1) * (kVec / 8);
  h.n_rowarr = n_rows;
  RVVLA_CUDA(cudaMalloc(&out->thr_info, (size_t)NT * 10 * sizeof(int)));
  RVVLA_CUDA(cudaMalloc(&out->veceor_ptr, (size_t)(n_eor + 1) * 4));
  RVVLA_CUDA(cudaMalloc(&out->scan_mask, (size_t)std::max<int64_t>(h.scan_mask_bytes, 4)));
  RVVLA_CUDA(cudaMalloc(&out->row_arr, (size_t)std::max<int64_t>(n_rows, 1) * 4));
  RVVLA_CUDA(cudaMalloc(&out->col_arr, (size_t)std::max<int64_t>(nvec * kVec, 1) * 4));
  RVVLA_CUDA(cudaMalloc(&out->vals_arr, (size_t)std::max<int64_t>(nvec * kVec, 1) * vb));
  // sentinel after the last thread's end-of-row vectors
  const uint32_t sentinel = (uint32_t)nvec;
  RVVLA_CUDA(cudaMemcpyAsync(out->veceor_ptr + n_eor, &sentinel, 4, cudaMemcpyHostToDevice, st));
  vhcc_fill_kernel<<<(unsigned)((NT + 127) / 128), 128, 0, st>>>(
      nvec, NT, m, nnz, src->Rst, s_bits.as<uint32_t>(), s_erow.as<int>(), s_eo.as<int64_t>(), s_ro.as<int64_t>(),
      out->veceor_ptr, reinterpret_cast<uint32_t*>(out->scan_mask), out->row_arr, out->thr_info);
  RVVLA_LAUNCHED("vhcc_fill_kernel");
  const int64_t total = nvec * kVec;
  if (total > 0) {
    const unsigned blocks = (unsigned)((total + 255) / 256);
    if (vb == 8) vhcc_pack_kernel<8><<<blocks, 256, 0, st>>>(total, nnz, src->Col, (const uint8_t*)src->Val, out->col_arr, (uint8_t*)out->vals_arr);
    else if (vb == 4) vhcc_pack_kernel<4><<<blocks, 256, 0, st>>>(total, nnz, src->Col, (const uint8_t*)src->Val, out->col_arr, (uint8_t*)out->vals_arr);
    else vhcc_pack_kernel<2><<<blocks, 256, 0, st>>>(total, nnz, src->Col, (const uint8_t*)src->Val, out->col_arr, (uint8_t*)out->vals_arr);
    RVVLA_LAUNCHED("vhcc_pack_kernel");
  }
  h.thr_info = out->thr_info; h.veceor_ptr = out->veceor_ptr; h.scan_mask = out->scan_mask;
  h.row_arr = out->row_arr; h.col_arr = out->col_arr; h.vals_arr = out->vals_arr;
  RVVLA_CUDA(cudaStreamSynchronize(st));
  return RVVLA_OK;
}

}  // namespace
}  // namespace rvvla

using namespace rvvla;

extern "C" {

int rvvla_vhcc_build(const rvvla_crs* src, int val_bytes, int64_t num_threads, rvvla_vhcc_owned* out, void* stream) {
  int rc = vhcc_build_impl(src, val_bytes, num_threads, out, as_stream(stream));
  if (rc && out) {
    std::string keep = rvvla_last_error();
    rvvla_vhcc_free(out);
    set_error(keep);
  }
  return rc;
}

void rvvla_vhcc_free(rvvla_vhcc_owned* h) {
  if (!h) return;
  cudaFree(h->thr_info);
  cudaFree(h->veceor_ptr);
  cudaFree(h->scan_mask);
  cudaFree(h->row_arr);
  cudaFree(h->col_arr);
  cudaFree(h->vals_arr);
  std::memset(h, 0, sizeof(*h));
}

int rvvla_vhcc_spmv_f64(const rvvla_vhcc* A, double alpha, const double* x, double beta, double* y, void* stream) {
  return vhcc_spmv_impl<double, double, double, double>(A, alpha, x, beta, y, as_stream(stream));
}

int rvvla_vhcc_spmv_f32(const rvvla_vhcc* A, float alpha, const float* x, float beta, float* y, void* stream) {
  return vhcc_spmv_impl<float, float, float, float>(A, alpha, x, beta, y, as_stream(stream));
}

}  // extern "C"
