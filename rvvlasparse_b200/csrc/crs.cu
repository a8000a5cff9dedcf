// crs.cu — y = alpha*A*x + beta*y for spMtxCRS (CSR) on sm_100a.
//
// Reference: sparse_mv<T, spMtxCRS, false> (src/scalar/spmv_mtx_crs.cpp:22-71)
// and the RVV version (src/rvv/spmv_mtx_crs.cpp:22-120): one sequential sum
// per row, y[i] = tmp*alpha + beta*y[i].
//
// B200 mapping: merge-path split (Merrill & Garland) of the item stream
// "row ends + nonzeros" into tiles of 256 threads x IPT items, so every CTA
// moves the same number of bytes whatever the row-length distribution
// (lognormal rows up to 4096 long are the design case).  Per tile:
//   1. coalesced loads of the tile's row ends and (values, columns) with
//      L2 evict-first, gather of x with L2 evict-last (x stays resident in the
//      126 MB L2 while the matrix streams past it); products go to shared
//      memory;
//   2. each thread walks IPT items of the merge path in shared memory;
//   3. a block-wide segmented scan (keys = row ids, non-decreasing) hands each
//      thread the partial sum of its first row from the threads before it;
//   4. the row that continues into the next tile leaves a (row, value) carry;
//      a second kernel adds carries in tile order (no float atomics, results
//      are bitwise reproducible run to run).
// The same kernels serve VNEC's L variant (merge-path CSR, vnec.cu).
//
// rvvla_crs_analyze picks the shared-memory-free lane-run kernel instead
// (crs_run.cuh; the warp-stream kernel of crs_stream.cuh on the same plan
// with RVVLA_CRS_KERNEL=stream) for every matrix with nonzeros: directly when
// no row is empty (plan kind 1), otherwise over the compacted non-empty rows
// with a map back to the row ids and a separate beta pass over the empty rows
// (kind 2).  Plan layouts (int32): kind 1 [wrow[nw], bits]; kind 2 [mc, me,
// wrow[nw], Rst_c[mc+1], row_map[mc], empty[me], bits] with plan_tiles = mc
// (nw follows from nz); bits = the row-start bitmap over the nonzeros,
// (nz + 31) / 32 words.
#include <algorithm>

#include "rvvla_internal.cuh"
#include "crs_merge.cuh"
#include "crs_run.cuh"
#include "crs_stream.cuh"
#include "scan.cuh"

#include <cstdlib>
#include <string>

namespace rvvla {

// Row-start bitmap: bit rst[r] for every row r with nonzeros.
__global__ void crs_run_bits_kernel(int m, const int* __restrict__ rst, uint32_t* __restrict__ bits) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < m && rst[r + 1] > rst[r]) atomicOr(bits + (rst[r] >> 5), 1u << (rst[r] & 31));
}


// Nonzeros per warp in the stream and lane-run kernels: 2048, halved (down
// to 256) while the matrix would give fewer than ~6 waves of 4736 warps (148
// SMs x 32 resident warps), so a medium-size matrix does not leave a large
// partial last wave.  A function of nz alone: the analysis and the SpMV
// agree on it.
int crs_warp_span(int64_t nz) {
  int E = 2048;
  while (E > 256 && nz < (int64_t)6 * 4736 * E) E >>= 1;
  return E;
}

__global__ void crs_stream_plan_kernel(int m, int nnz, const int* __restrict__ Rst, int E, int nwarps,
                                       int* __restrict__ wrow, int* __restrict__ any_empty) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < nwarps) {
    const int e = t * E;  // largest r with Rst[r] <= e
    int lo = 0, hi = m + 1;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (Rst[mid] <= e) lo = mid;
      else hi = mid;
    }
    wrow[t] = lo;
  }
  if (t < m && Rst[t + 1] == Rst[t]) atomicOr(any_empty, 1);
}

// kind 2: non-empty rows compacted (scan of the non-empty flags)
__global__ void crs_nonempty_flags_kernel(int m, const int* __restrict__ Rst, int64_t* __restrict__ flag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) flag[i] = Rst[i + 1] > Rst[i] ? 1 : 0;
}

__global__ void crs_compact_kernel(int m, int nnz, const int* __restrict__ Rst, const int64_t* __restrict__ pos,
                                   int* __restrict__ rst_c, int* __restrict__ row_map, int* __restrict__ empty) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) {
    const int p = (int)pos[i];
    if (Rst[i + 1] > Rst[i]) {
      rst_c[p] = Rst[i];
      row_map[p] = i;
    } else {
      empty[i - p] = i;
    }
  }
  if (i == 0) rst_c[pos[m]] = nnz;
}

template <class X>
__global__ void crs_empty_rows_kernel(int me, const int* __restrict__ empty, X* __restrict__ y, X beta) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < me) {
    const int r = empty[i];
    y[r] = (beta == X(0)) ? X(0) : beta * y[r];
  }
}

__global__ void merge_plan_kernel(int m, int nnz, const int* __restrict__ Rst, int tile_items, int ntiles,
                                  int* __restrict__ plan) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t > ntiles) return;
  const long long items = (long long)m + nnz;
  const int diag = (int)min((long long)t * tile_items, items);
  int lo = max(diag - nnz, 0), hi = min(diag, m);
  while (lo < hi) {
    const int piv = (lo + hi) >> 1;
    if (Rst[piv + 1] <= diag - piv - 1) lo = piv + 1;
    else hi = piv;
  }
  plan[2 * t] = lo;
  plan[2 * t + 1] = diag - lo;
}

// The kernel for plan kinds 1 and 2 (a tuning knob read once).
bool crs_use_stream_kernel() {
  static const bool stream = [] {
    const char* e = std::getenv("RVVLA_CRS_KERNEL");
    return e && std::string(e) == "stream";
  }();
  return stream;
}

int64_t crs_tiles(int64_t m, int64_t nz, int ipt) {
  const int64_t tile = (int64_t)kMergeBlock * ipt;
  return (m + nz + tile - 1) / tile;
}

int crs_validate(const rvvla_crs* A, const void* x, const void* y) {
  if (!A) return fail(RVVLA_ERR_INVALID_ARG, "crs: null descriptor");
  if (A->m < 0 || A->n < 0 || A->nz < 0) return fail(RVVLA_ERR_INVALID_ARG, "crs: negative size");
  if (A->m + A->nz >= (int64_t)INT32_MAX - 65536) return fail(RVVLA_ERR_TOO_LARGE, "crs: m + nz exceeds int32 merge-path range");
  if (A->m > 0 && !A->Rst) return fail(RVVLA_ERR_INVALID_ARG, "crs: null Rst");
  if (A->nz > 0 && (!A->Col || !A->Val)) return fail(RVVLA_ERR_INVALID_ARG, "crs: null Col/Val");
  if (A->m > 0 && !y) return fail(RVVLA_ERR_INVALID_ARG, "crs: null y");
  if (A->nz > 0 && !x) return fail(RVVLA_ERR_INVALID_ARG, "crs: null x");
  return RVVLA_OK;
}

int crs_plan_launch(int64_t m, int64_t nz, const int32_t* Rst, int ipt, int32_t* plan, cudaStream_t st) {
  const int64_t nt = crs_tiles(m, nz, ipt);
  const int threads = 256;
  const int64_t blocks = (nt + 1 + threads - 1) / threads;
  merge_plan_kernel<<<(unsigned)blocks, threads, 0, st>>>((int)m, (int)nz, Rst, kMergeBlock * ipt, (int)nt, plan);
  RVVLA_LAUNCHED("merge_plan_kernel");
  return RVVLA_OK;
}

// perm/pval (the adjoint): value k of A is pval[perm[k]]; needs an analysed
// plan (kinds 1 and 2) when A has nonzeros.
// dot_part (the solvers): the lane-run kernel also writes one partial of
// x^T (y - beta y) / alpha per warp (see crs_run_kernel), *nparts of them
// (at most dot_cap); needs an analysed plan.
template <class V, class X, class Ac, class P, class CT, int IPT>
int crs_spmv_impl(const rvvla_crs* A, X alpha, const X* x, X beta, X* y, cudaStream_t st,
                  const int32_t* perm = nullptr, const V* pval = nullptr, CT* dot_part = nullptr,
                  int64_t dot_cap = 0, int64_t* nparts = nullptr) {
  int rc = crs_validate(A, x, y);
  if (rc) return rc;
  if (nparts) *nparts = 0;
  if (A->m == 0) return RVVLA_OK;
  if ((perm || dot_part) && A->nz > 0 && !(A->plan && (A->plan_kind == 1 || A->plan_kind == 2)))
    return fail(RVVLA_ERR_INVALID_ARG, "crs: this product needs an analysed plan (rvvla_crs_analyze)");
  if (A->plan && (A->plan_kind == 1 || A->plan_kind == 2)) {  // shared-memory-free stream kernel
    // kind 1: plan_tiles = warps, all rows; kind 2: plan_tiles = number of
    // non-empty rows, the warps run over the compacted rows
    const int E = crs_warp_span(A->nz);
    const int64_t nw = (A->nz + E - 1) / E;
    if (A->nz == 0 || (A->plan_kind == 1 && A->plan_tiles != nw) ||
        (A->plan_kind == 2 && (A->plan_tiles <= 0 || A->plan_tiles > A->m)))
      return fail(RVVLA_ERR_INVALID_ARG, "crs: stream plan was built for a different matrix");
    const int32_t* wrow = A->plan;
    const int32_t* rst = A->Rst;
    const int32_t* row_map = nullptr;
    const uint32_t* bits = reinterpret_cast<const uint32_t*>(A->plan + nw);
    int mr = (int)A->m;
    if (A->plan_kind == 2) {
      const int mc = (int)A->plan_tiles, me = (int)(A->m - A->plan_tiles);
      wrow = A->plan + 2;
      rst = wrow + nw;
      row_map = rst + mc + 1;
      const int32_t* empty = row_map + mc;
      bits = reinterpret_cast<const uint32_t*>(empty + me);
      mr = mc;
      if (me > 0) {
        crs_empty_rows_kernel<X><<<(unsigned)((me + 255) / 256), 256, 0, st>>>(me, empty, y, beta);
        RVVLA_LAUNCHED("crs_empty_rows_kernel");
      }
    }
    Scratch sc;
    const size_t row_bytes = ((size_t)(2 * nw) * sizeof(int32_t) + 255) / 256 * 256;
    RVVLA_CUDA(sc.alloc(row_bytes + (size_t)(2 * nw) * sizeof(CT), st));
    int32_t* crow = sc.as<int32_t>();
    CT* cval = (CT*)(sc.as<char>() + row_bytes);
    const unsigned blocks = (unsigned)((nw * 32 + 255) / 256);
    if (dot_part) {
      if (nw > dot_cap) return fail(RVVLA_ERR_TOO_LARGE, "crs: dot partial buffer too small");
      *nparts = nw;
      const bool vec = (uintptr_t)A->Col % 16 == 0 && (uintptr_t)A->Val % 16 == 0;
      if (vec)
        crs_run_kernel<V, X, Ac, CT, true, false, true><<<blocks, 256, 0, st>>>(
            mr, (int)A->nz, E, (int)nw, rst, bits, A->Col, (const V*)A->Val, x, y, alpha, beta, wrow, crow, cval,
            row_map, nullptr, dot_part);
      else
        crs_run_kernel<V, X, Ac, CT, false, false, true><<<blocks, 256, 0, st>>>(
            mr, (int)A->nz, E, (int)nw, rst, bits, A->Col, (const V*)A->Val, x, y, alpha, beta, wrow, crow, cval,
            row_map, nullptr, dot_part);
      RVVLA_LAUNCHED("crs_run_kernel");
    } else if (perm) {
      const bool vec = (uintptr_t)A->Col % 16 == 0 && (uintptr_t)perm % 16 == 0;
      if (vec)
        crs_run_kernel<V, X, Ac, CT, true, true><<<blocks, 256, 0, st>>>(
            mr, (int)A->nz, E, (int)nw, rst, bits, A->Col, pval, x, y, alpha, beta, wrow, crow, cval, row_map,
            perm);
      else
        crs_run_kernel<V, X, Ac, CT, false, true><<<blocks, 256, 0, st>>>(
            mr, (int)A->nz, E, (int)nw, rst, bits, A->Col, pval, x, y, alpha, beta, wrow, crow, cval, row_map,
            perm);
      RVVLA_LAUNCHED("crs_run_kernel");
    } else if (crs_use_stream_kernel()) {
      crs_stream_kernel<V, X, Ac, CT><<<blocks, 256, 0, st>>>(mr, (int)A->nz, E, (int)nw, rst, A->Col,
                                                              (const V*)A->Val, x, y, alpha, beta, wrow, crow, cval,
                                                              row_map);
      RVVLA_LAUNCHED("crs_stream_kernel");
    } else {
      const bool vec = (uintptr_t)A->Col % 16 == 0 && (uintptr_t)A->Val % 16 == 0;
      if (vec)
        crs_run_kernel<V, X, Ac, CT, true><<<blocks, 256, 0, st>>>(mr, (int)A->nz, E, (int)nw, rst, bits,
                                                                   A->Col, (const V*)A->Val, x, y, alpha, beta, wrow,
                                                                   crow, cval, row_map);
      else
        crs_run_kernel<V, X, Ac, CT, false><<<blocks, 256, 0, st>>>(mr, (int)A->nz, E, (int)nw, rst, bits,
                                                                    A->Col, (const V*)A->Val, x, y, alpha, beta, wrow,
                                                                    crow, cval, row_map);
      RVVLA_LAUNCHED("crs_run_kernel");
    }
    crs_stream_fixup_kernel<X, CT><<<(unsigned)((2 * nw + 255) / 256), 256, 0, st>>>((int)(2 * nw), crow, cval, y,
                                                                                       alpha, beta, row_map);
    RVVLA_LAUNCHED("crs_stream_fixup_kernel");
    return RVVLA_OK;
  }
  const int64_t nt = crs_tiles(A->m, A->nz, IPT);
  const int32_t* plan = A->plan;
  if (plan && A->plan_tiles != nt)
    return fail(RVVLA_ERR_INVALID_ARG, "crs: plan was built for a different size or value type");
  const size_t plan_bytes = plan ? 0 : (size_t)(2 * (nt + 1)) * sizeof(int32_t);
  const size_t row_off = (plan_bytes + 255) / 256 * 256;
  const size_t val_off = row_off + ((size_t)nt * sizeof(int32_t) + 255) / 256 * 256;
  Scratch sc;
  RVVLA_CUDA(sc.alloc(val_off + (size_t)nt * sizeof(CT), st));
  char* base = sc.as<char>();
  if (!plan) {
    rc = crs_plan_launch(A->m, A->nz, A->Rst, IPT, (int32_t*)base, st);
    if (rc) return rc;
    plan = (const int32_t*)base;
  }
  int32_t* crow = (int32_t*)(base + row_off);
  CT* cval = (CT*)(base + val_off);
  prefer_shared(merge_spmv_kernel<V, X, Ac, P, CT, IPT>);
  merge_spmv_kernel<V, X, Ac, P, CT, IPT><<<(unsigned)nt, kMergeBlock, 0, st>>>(
      (int)A->m, (int)A->nz, A->Rst, A->Col, (const V*)A->Val, x, y, alpha, beta, plan, crow, cval);
  RVVLA_LAUNCHED("merge_spmv_kernel");
  merge_fixup_kernel<X, CT><<<(unsigned)((nt + 255) / 256), 256, 0, st>>>((int)nt, (int)A->m, crow, cval, y, alpha);
  RVVLA_LAUNCHED("merge_fixup_kernel");
  return RVVLA_OK;
}

// q = A p with the fused dot (alpha 1, beta 0): part[0..*nparts) sum to
// p^T A p; used by the solvers.
int crs_spmv_dot_f64(const rvvla_crs* A, const double* p, double* q, double* part, int64_t cap, int64_t* nparts,
                     cudaStream_t st) {
  return crs_spmv_impl<double, double, double, double, double, MergeCfg<double>::IPT>(A, 1.0, p, 0.0, q, st, nullptr,
                                                                                      nullptr, part, cap, nparts);
}
int crs_spmv_dot_f32(const rvvla_crs* A, const float* p, float* q, float* part, int64_t cap, int64_t* nparts,
                     cudaStream_t st) {
  return crs_spmv_impl<float, float, float, float, float, MergeCfg<float>::IPT>(A, 1.0f, p, 0.0f, q, st, nullptr,
                                                                               nullptr, part, cap, nparts);
}
int64_t crs_warp_count(int64_t nz) {
  const int E = crs_warp_span(nz);
  return (nz + E - 1) / E;
}

}  // namespace rvvla

using namespace rvvla;

extern "C" {

int64_t rvvla_crs_plan_len(int64_t m, int64_t nz, int dtype) {
  const int ipt = dtype == RVVLA_F64 ? MergeCfg<double>::IPT : MergeCfg<float>::IPT;
  const int64_t nw = (nz + 255) / 256;  // the most warps any span gives
  return std::max<int64_t>(2 * (crs_tiles(m, nz, ipt) + 1), 3 * m + nw + 3 + (nz + 31) / 32);
}

int rvvla_crs_analyze(const rvvla_crs* A, int dtype, int32_t* plan, int64_t* plan_tiles, int32_t* plan_kind,
                      void* stream) {
  if (!A || !plan || !plan_tiles || !plan_kind) return fail(RVVLA_ERR_INVALID_ARG, "crs_analyze: null argument");
  if (A->m < 0 || A->nz < 0 || (A->m > 0 && !A->Rst)) return fail(RVVLA_ERR_INVALID_ARG, "crs_analyze: bad matrix");
  if (A->m + A->nz >= (int64_t)INT32_MAX - 65536) return fail(RVVLA_ERR_TOO_LARGE, "crs_analyze: too large");
  const int ipt = dtype == RVVLA_F64 ? MergeCfg<double>::IPT : MergeCfg<float>::IPT;
  *plan_tiles = 0;
  *plan_kind = 0;
  if (A->m == 0) return RVVLA_OK;
  cudaStream_t st = as_stream(stream);
  if (A->nz > 0) {
    const int E = crs_warp_span(A->nz);
    const int64_t nw = (A->nz + E - 1) / E;
    Scratch flag;
    RVVLA_CUDA(flag.alloc(sizeof(int), st));
    RVVLA_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int), st));
    const int64_t n = std::max<int64_t>(nw, A->m);
    crs_stream_plan_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>((int)A->m, (int)A->nz, A->Rst, E,
                                                                         (int)nw, plan, flag.as<int>());
    RVVLA_LAUNCHED("crs_stream_plan_kernel");
    int any_empty = 1;
    RVVLA_CUDA(cudaMemcpyAsync(&any_empty, flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    RVVLA_CUDA(cudaStreamSynchronize(st));
    if (!any_empty) {
      uint32_t* bits = reinterpret_cast<uint32_t*>(plan + nw);
      RVVLA_CUDA(cudaMemsetAsync(bits, 0, (size_t)((A->nz + 31) / 32) * sizeof(uint32_t), st));
      crs_run_bits_kernel<<<(unsigned)((A->m + 255) / 256), 256, 0, st>>>((int)A->m, A->Rst, bits);
      RVVLA_LAUNCHED("crs_run_bits_kernel");
      RVVLA_CUDA(cudaStreamSynchronize(st));
      *plan_tiles = nw;
      *plan_kind = 1;
      return RVVLA_OK;
    }
    // kind 2: compact the non-empty rows, then split the warps over them
    Scratch s_flag, s_pos;
    RVVLA_CUDA(s_flag.alloc((size_t)A->m * sizeof(int64_t), st));
    RVVLA_CUDA(s_pos.alloc((size_t)(A->m + 1) * sizeof(int64_t), st));
    const unsigned mb = (unsigned)((A->m + 255) / 256);
    crs_nonempty_flags_kernel<<<mb, 256, 0, st>>>((int)A->m, A->Rst, s_flag.as<int64_t>());
    RVVLA_LAUNCHED("crs_nonempty_flags_kernel");
    int rc = exclusive_scan_i64(s_flag.as<int64_t>(), s_pos.as<int64_t>(), A->m, st);
    if (rc) return rc;
    int64_t mc = 0;
    RVVLA_CUDA(cudaMemcpyAsync(&mc, s_pos.as<int64_t>() + A->m, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    RVVLA_CUDA(cudaStreamSynchronize(st));
    const int64_t me = A->m - mc;
    int32_t* wrow = plan + 2;
    int32_t* rst_c = wrow + nw;
    int32_t* row_map = rst_c + mc + 1;
    int32_t* empty = row_map + mc;
    crs_compact_kernel<<<mb, 256, 0, st>>>((int)A->m, (int)A->nz, A->Rst, s_pos.as<int64_t>(), rst_c, row_map, empty);
    RVVLA_LAUNCHED("crs_compact_kernel");
    crs_stream_plan_kernel<<<(unsigned)((nw + 255) / 256), 256, 0, st>>>((int)mc, (int)A->nz, rst_c, E,
                                                                         (int)nw, wrow, flag.as<int>());
    RVVLA_LAUNCHED("crs_stream_plan_kernel");
    uint32_t* bits = reinterpret_cast<uint32_t*>(empty + me);
    RVVLA_CUDA(cudaMemsetAsync(bits, 0, (size_t)((A->nz + 31) / 32) * sizeof(uint32_t), st));
    if (mc > 0) {
      crs_run_bits_kernel<<<(unsigned)((mc + 255) / 256), 256, 0, st>>>((int)mc, rst_c, bits);
      RVVLA_LAUNCHED("crs_run_bits_kernel");
    }
    const int32_t hdr[2] = {(int32_t)mc, (int32_t)me};
    RVVLA_CUDA(cudaMemcpyAsync(plan, hdr, sizeof(hdr), cudaMemcpyHostToDevice, st));
    RVVLA_CUDA(cudaStreamSynchronize(st));
    *plan_tiles = mc;
    *plan_kind = 2;
    return RVVLA_OK;
  }
  *plan_tiles = crs_tiles(A->m, A->nz, ipt);
  *plan_kind = 0;
  return crs_plan_launch(A->m, A->nz, A->Rst, ipt, plan, st);
}

int rvvla_crs_spmv_f64(const rvvla_crs* A, double alpha, const double* x, double beta, double* y, void* stream) {
  return crs_spmv_impl<double, double, double, double, double, MergeCfg<double>::IPT>(A, alpha, x, beta, y,
                                                                                      as_stream(stream));
}

int rvvla_crs_spmv_f32(const rvvla_crs* A, float alpha, const float* x, float beta, float* y, void* stream) {
  return crs_spmv_impl<float, float, float, float, float, MergeCfg<float>::IPT>(A, alpha, x, beta, y,
                                                                               as_stream(stream));
}

int rvvla_spmv_adjoint_x_values_f64(const rvvla_transpose* T, const double* Val, double alpha, const double* g,
                                    double beta, double* dx, void* stream) {
  if (!T || T->val_bytes != 8) return fail(RVVLA_ERR_INVALID_ARG, "spmv_adjoint_x_values_f64: needs an fp64 transpose");
  if (T->AT.nz > 0 && (!T->perm || !Val)) return fail(RVVLA_ERR_INVALID_ARG, "spmv_adjoint_x_values_f64: null array");
  return crs_spmv_impl<double, double, double, double, double, MergeCfg<double>::IPT>(&T->AT, alpha, g, beta, dx,
                                                                                      as_stream(stream), T->perm, Val);
}

int rvvla_spmv_adjoint_x_values_f32(const rvvla_transpose* T, const float* Val, float alpha, const float* g,
                                    float beta, float* dx, void* stream) {
  if (!T || T->val_bytes != 4) return fail(RVVLA_ERR_INVALID_ARG, "spmv_adjoint_x_values_f32: needs an fp32 transpose");
  if (T->AT.nz > 0 && (!T->perm || !Val)) return fail(RVVLA_ERR_INVALID_ARG, "spmv_adjoint_x_values_f32: null array");
  return crs_spmv_impl<float, float, float, float, float, MergeCfg<float>::IPT>(&T->AT, alpha, g, beta, dx,
                                                                               as_stream(stream), T->perm, Val);
}

int rvvla_crs_spmv_mixed(const rvvla_crs* A, int val_type, float alpha, const float* x, float beta, float* y,
                         void* stream) {
  if (val_type == RVVLA_F32)
    return crs_spmv_impl<float, float, CompF32, float, double, MergeCfg<float>::IPT>(A, alpha, x, beta, y,
                                                                                    as_stream(stream));
  if (val_type == RVVLA_BF16)
    return crs_spmv_impl<__nv_bfloat16, float, CompF32, float, double, MergeCfg<float>::IPT>(A, alpha, x, beta, y,
                                                                                            as_stream(stream));
  return fail(RVVLA_ERR_INVALID_ARG, "crs_spmv_mixed: val_type must be RVVLA_F32 or RVVLA_BF16");
}

}  // extern "C"
