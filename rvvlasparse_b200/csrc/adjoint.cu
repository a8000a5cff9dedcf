// adjoint.cu — the adjoint of CRS SpMV (no reference counterpart).
//
// For y = alpha * A(v) x with A's sparsity fixed and values v:
//   dx = A^T g        through a transposed CRS built on the GPU once per
//                     pattern (rvvla_csr_transpose); the product itself runs
//                     the CRS SpMV kernels on A^T (row streaming, no atomics,
//                     deterministic);
//   dv[k] = g[row(k)] * x[Col[k]]   sampled on A's pattern (SDDMM).
// When the values change but the pattern does not, rvvla_csr_transpose_values
// re-gathers A^T's values through the stored permutation.
//
// Transpose: row index of every nonzero (warp per row), a stable radix sort
// of (column, nonzero index) pairs, row pointers of A^T from the boundaries
// of the sorted columns, then gathers of row indices and values through the
// permutation.  Inside a column the entries keep A's order (ascending rows),
// as a counting-sort transpose would produce.
#include <cub/device/device_radix_sort.cuh>

#include <cstring>
#include <string>

#include "rvvla_internal.cuh"

namespace rvvla {
namespace {

__global__ void row_expand_kernel(int64_t m, const int* __restrict__ Rst, int* __restrict__ rowid) {
  const int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= m) return;
  const int b = Rst[r], e = Rst[r + 1];
  for (int k = b + lane; k < e; k += 32) rowid[k] = (int)r;
}

__global__ void iota_kernel(int64_t n, int* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (int)i;
}

// RstT[c] = first sorted position whose column is >= c (c = 0..ncols).
__global__ void tr_bounds_kernel(int64_t nz, int64_t ncols, const uint32_t* __restrict__ skey,
                                 int* __restrict__ RstT) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k > nz) return;
  const int64_t prev = (k == 0) ? -1 : (int64_t)skey[k - 1];
  const int64_t cur = (k == nz) ? ncols : (int64_t)skey[k];
  for (int64_t c = prev + 1; c <= cur; ++c) RstT[c] = (int)k;
}

template <int VB>
struct Word;
template <>
struct Word<8> { using T = unsigned long long; };
template <>
struct Word<4> { using T = unsigned int; };
template <>
struct Word<2> { using T = unsigned short; };

template <int VB>
__global__ void tr_gather_kernel(int64_t nz, const int* __restrict__ perm, const int* __restrict__ rowid,
                                 const void* __restrict__ val, int* __restrict__ ColT, void* __restrict__ ValT) {
  using W = typename Word<VB>::T;
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nz) return;
  const int p = perm[k];
  if (ColT) ColT[k] = rowid[p];
  if (val) static_cast<W*>(ValT)[k] = static_cast<const W*>(val)[p];
}

constexpr int kSdThreads = 256;
constexpr int kSdRows = 256;  // rows per CTA
constexpr int kSdU = 4;       // nonzeros per thread in flight

// dv[k] = g[row(k)] * x[Col[k]]: a CTA per 256 consecutive rows, their row
// pointers staged in shared memory (no search in global memory); each thread
// takes every 256th nonzero of the CTA's range, finds its row by binary
// search over the staged pointers and keeps 4 nonzeros' loads in flight.
template <class T>
__global__ void __launch_bounds__(kSdThreads)
sddmm_kernel(int64_t m, const int* __restrict__ Rst, const int* __restrict__ Col, const T* __restrict__ g,
             const T* __restrict__ x, T* __restrict__ dv) {
  __shared__ int win[kSdRows + 1];
  const int64_t r0 = (int64_t)blockIdx.x * kSdRows;
  const int nr = (int)min((int64_t)kSdRows, m - r0);
  for (int i = threadIdx.x; i <= nr; i += kSdThreads) win[i] = Rst[r0 + i];
  __syncthreads();
  const int kb = win[0], ke = win[nr];
  const uint64_t pf = policy_evict_first(), pl = policy_evict_last();
  for (int k0 = kb + (int)threadIdx.x; k0 < ke; k0 += kSdU * kSdThreads) {
    int c[kSdU];
    T gv[kSdU];
#pragma unroll
    for (int u = 0; u < kSdU; ++u) {
      const int k = min(k0 + u * kSdThreads, ke - 1);
      int lo = 0, hi = nr - 1;  // largest j with win[j] <= k
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (win[mid] <= k) lo = mid;
        else hi = mid - 1;
      }
      c[u] = ld_stream(Col + k, pf);
      gv[u] = g[r0 + lo];
    }
#pragma unroll
    for (int u = 0; u < kSdU; ++u) {
      const int k = k0 + u * kSdThreads;
      const T xv = ld_keep(x + c[u], pl);
      if (k < ke) dv[k] = gv[u] * xv;
    }
  }
}

int transpose_impl(const rvvla_crs* A, int vb, rvvla_transpose_owned* out, cudaStream_t st) {
  if (!A || !out) return fail(RVVLA_ERR_INVALID_ARG, "csr_transpose: null argument");
  std::memset(out, 0, sizeof(*out));
  if (vb != 8 && vb != 4 && vb != 2) return fail(RVVLA_ERR_INVALID_ARG, "csr_transpose: val_bytes must be 8, 4 or 2");
  const int64_t m = A->m, n = A->n, nz = A->nz;
  if (m < 0 || n < 0 || nz < 0) return fail(RVVLA_ERR_INVALID_ARG, "csr_transpose: bad sizes");
  if (nz >= INT32_MAX || m >= INT32_MAX || n >= INT32_MAX)
    return fail(RVVLA_ERR_TOO_LARGE, "csr_transpose: sizes beyond int32");
  if (m > 0 && !A->Rst) return fail(RVVLA_ERR_INVALID_ARG, "csr_transpose: null Rst");
  if (nz > 0 && !A->Col) return fail(RVVLA_ERR_INVALID_ARG, "csr_transpose: null Col");
  const bool with_vals = A->Val != nullptr;
  RVVLA_CUDA(cudaMalloc(&out->Rst, (size_t)(n + 1) * sizeof(int)));
  RVVLA_CUDA(cudaMalloc(&out->Col, (size_t)std::max<int64_t>(nz, 1) * sizeof(int)));
  RVVLA_CUDA(cudaMalloc(&out->perm, (size_t)std::max<int64_t>(nz, 1) * sizeof(int)));
  RVVLA_CUDA(cudaMalloc(&out->Val, (size_t)std::max<int64_t>(nz, 1) * vb));
  if (nz > 0) {
    Scratch s_row, s_idx, s_key, s_tmp;
    RVVLA_CUDA(s_row.alloc((size_t)nz * sizeof(int), st));
    RVVLA_CUDA(s_idx.alloc((size_t)nz * sizeof(int), st));
    RVVLA_CUDA(s_key.alloc((size_t)nz * sizeof(uint32_t), st));
    row_expand_kernel<<<(unsigned)((m * 32 + 255) / 256), 256, 0, st>>>(m, A->Rst, s_row.as<int>());
    RVVLA_LAUNCHED("row_expand_kernel");
    iota_kernel<<<(unsigned)((nz + 255) / 256), 256, 0, st>>>(nz, s_idx.as<int>());
    RVVLA_LAUNCHED("iota_kernel");
    int end_bit = 1;
    while (end_bit < 32 && (int64_t(1) << end_bit) < n) end_bit++;
    size_t tmp_bytes = 0;
    const uint32_t* keys_in = reinterpret_cast<const uint32_t*>(A->Col);
    RVVLA_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys_in, s_key.as<uint32_t>(), s_idx.as<int>(),
                                               out->perm, (int)nz, 0, end_bit, st));
    RVVLA_CUDA(s_tmp.alloc(tmp_bytes, st));
    RVVLA_CUDA(cub::DeviceRadixSort::SortPairs(s_tmp.p, tmp_bytes, keys_in, s_key.as<uint32_t>(), s_idx.as<int>(),
                                               out->perm, (int)nz, 0, end_bit, st));
    count_launch(3);
    tr_bounds_kernel<<<(unsigned)((nz + 1 + 255) / 256), 256, 0, st>>>(nz, n, s_key.as<uint32_t>(), out->Rst);
    RVVLA_LAUNCHED("tr_bounds_kernel");
    const unsigned blocks = (unsigned)((nz + 255) / 256);
    const void* vals = with_vals ? A->Val : nullptr;
    if (vb == 8) tr_gather_kernel<8><<<blocks, 256, 0, st>>>(nz, out->perm, s_row.as<int>(), vals, out->Col, out->Val);
    else if (vb == 4) tr_gather_kernel<4><<<blocks, 256, 0, st>>>(nz, out->perm, s_row.as<int>(), vals, out->Col, out->Val);
    else tr_gather_kernel<2><<<blocks, 256, 0, st>>>(nz, out->perm, s_row.as<int>(), vals, out->Col, out->Val);
    RVVLA_LAUNCHED("tr_gather_kernel");
  } else {
    RVVLA_CUDA(cudaMemsetAsync(out->Rst, 0, (size_t)(n + 1) * sizeof(int), st));
  }
  rvvla_transpose& h = out->h;
  h.AT.m = n; h.AT.n = m; h.AT.nz = nz;
  h.AT.Rst = out->Rst; h.AT.Col = out->Col; h.AT.Val = out->Val;
  h.perm = out->perm;
  h.val_bytes = vb;
  // analysis plan of A^T for the CRS kernels (value type decides the tile)
  if (n > 0) {
    const int dt = (vb == 8) ? RVVLA_F64 : RVVLA_F32;
    const int64_t plen = rvvla_crs_plan_len(n, nz, dt);
    RVVLA_CUDA(cudaMalloc(&out->plan, (size_t)std::max<int64_t>(plen, 1) * sizeof(int32_t)));
    int64_t tiles = 0;
    int32_t kind = 0;
    const int rc = rvvla_crs_analyze(&h.AT, dt, out->plan, &tiles, &kind, st);
    if (rc) return rc;
    h.AT.plan = out->plan; h.AT.plan_tiles = tiles; h.AT.plan_kind = kind;
  }
  RVVLA_CUDA(cudaStreamSynchronize(st));
  return RVVLA_OK;
}

int transpose_check(const rvvla_transpose* T) {
  if (!T) return fail(RVVLA_ERR_INVALID_ARG, "adjoint: null transpose");
  if (T->AT.m < 0 || T->AT.n < 0 || T->AT.nz < 0) return fail(RVVLA_ERR_INVALID_ARG, "adjoint: bad sizes");
  if (T->AT.nz > 0 && (!T->perm || !T->AT.Col)) return fail(RVVLA_ERR_INVALID_ARG, "adjoint: null arrays");
  return RVVLA_OK;
}

template <class T>
int sddmm_impl(const rvvla_crs* A, const T* g, const T* x, T* dv, cudaStream_t st) {
  if (!A) return fail(RVVLA_ERR_INVALID_ARG, "sddmm: null descriptor");
  if (A->m < 0 || A->n < 0 || A->nz < 0) return fail(RVVLA_ERR_INVALID_ARG, "sddmm: bad sizes");
  if (A->nz == 0) return RVVLA_OK;
  if (!A->Rst || !A->Col || !g || !x || !dv) return fail(RVVLA_ERR_INVALID_ARG, "sddmm: null array");
  const int64_t blocks = (A->m + kSdRows - 1) / kSdRows;
  sddmm_kernel<T><<<(unsigned)blocks, kSdThreads, 0, st>>>(A->m, A->Rst, A->Col, g, x, dv);
  RVVLA_LAUNCHED("sddmm_kernel");
  return RVVLA_OK;
}

}  // namespace
}  // namespace rvvla

using namespace rvvla;

extern "C" {

int rvvla_csr_transpose(const rvvla_crs* A, int val_bytes, rvvla_transpose_owned* out, void* stream) {
  const int rc = transpose_impl(A, val_bytes, out, as_stream(stream));
  if (rc && out) {
    std::string keep = rvvla_last_error();
    rvvla_csr_transpose_free(out);
    set_error(keep);
  }
  return rc;
}

void rvvla_csr_transpose_free(rvvla_transpose_owned* h) {
  if (!h) return;
  void* ptrs[] = {h->Rst, h->Col, h->perm, h->plan, h->Val};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  std::memset(h, 0, sizeof(*h));
}

int rvvla_csr_transpose_values(const rvvla_transpose* T, const void* Val, void* ValT, void* stream) {
  int rc = transpose_check(T);
  if (rc) return rc;
  if (T->AT.nz == 0) return RVVLA_OK;
  if (!Val || !ValT) return fail(RVVLA_ERR_INVALID_ARG, "csr_transpose_values: null array");
  cudaStream_t st = as_stream(stream);
  const unsigned blocks = (unsigned)((T->AT.nz + 255) / 256);
  switch (T->val_bytes) {
    case 8: tr_gather_kernel<8><<<blocks, 256, 0, st>>>(T->AT.nz, T->perm, nullptr, Val, nullptr, ValT); break;
    case 4: tr_gather_kernel<4><<<blocks, 256, 0, st>>>(T->AT.nz, T->perm, nullptr, Val, nullptr, ValT); break;
    case 2: tr_gather_kernel<2><<<blocks, 256, 0, st>>>(T->AT.nz, T->perm, nullptr, Val, nullptr, ValT); break;
    default: return fail(RVVLA_ERR_INVALID_ARG, "csr_transpose_values: val_bytes must be 8, 4 or 2");
  }
  RVVLA_LAUNCHED("tr_gather_kernel");
  return RVVLA_OK;
}

int rvvla_spmv_adjoint_x_f64(const rvvla_transpose* T, double alpha, const double* g, double beta, double* dx,
                             void* stream) {
  int rc = transpose_check(T);
  if (rc) return rc;
  if (T->val_bytes != 8) return fail(RVVLA_ERR_INVALID_ARG, "spmv_adjoint_x_f64: transpose holds non-fp64 values");
  return rvvla_crs_spmv_f64(&T->AT, alpha, g, beta, dx, stream);
}

int rvvla_spmv_adjoint_x_f32(const rvvla_transpose* T, float alpha, const float* g, float beta, float* dx,
                             void* stream) {
  int rc = transpose_check(T);
  if (rc) return rc;
  if (T->val_bytes != 4) return fail(RVVLA_ERR_INVALID_ARG, "spmv_adjoint_x_f32: transpose holds non-fp32 values");
  return rvvla_crs_spmv_f32(&T->AT, alpha, g, beta, dx, stream);
}

int rvvla_sddmm_values_f64(const rvvla_crs* A, const double* g, const double* x, double* dvalues, void* stream) {
  return sddmm_impl<double>(A, g, x, dvalues, as_stream(stream));
}

int rvvla_sddmm_values_f32(const rvvla_crs* A, const float* g, const float* x, float* dvalues, void* stream) {
  return sddmm_impl<float>(A, g, x, dvalues, as_stream(stream));
}

}  // extern "C"
