// vnec.cu — spMtxVNEC on sm_100a (variants S, D, L of
// src/rvv/spmv_mtx_vnec.cpp:78-586; selection include/VNEC.h:218-226).
//
//   L (merge-path CSR, :448-586): the builder analyses the source CRS and the
//     SpMV runs the CRS lane-run kernel of crs.cu on that plan (the product is
//     the CRS one; the reference's merge path is only its CPU split); without
//     a plan, the merge-path kernels of crs.cu with the structure's thread
//     coordinates as tile boundaries (one CTA per VNEC thread) when a thread
//     holds at most one tile of items, else a fresh merge-path split;
//   D (:282-446): one CTA per VNEC thread; its compacted x (use_x_indices)
//     is staged in shared memory, each row's nLanes-wide column groups are
//     read as val_align windows (lanes = (group, lane) pairs, coalesced), the
//     row that continues into the next thread leaves a carry merged in thread
//     order by the merge-path fix-up kernel;
//   S (:78-280): one CTA per VNEC thread; compacted x in shared memory;
//     cross-row groups of nLanes rows (lane k of a group owns row k),
//     in-row rows one warp each.
// Every row is written once with alpha/beta (D and L also through carries).
#include <algorithm>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "crs_merge.cuh"
#include "rvvla_internal.cuh"

namespace rvvla {
namespace {

constexpr int kVnecThreads = 256;

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
  return v;
}

template <class X>
__device__ void stage_x(X* xx, const int* ux, int nec, int nL, const X* x) {
  const uint64_t pl = policy_evict_last();
  for (int j = threadIdx.x; j < nec + nL; j += blockDim.x) xx[j] = (j < nec) ? ld_keep(x + ux[j], pl) : X(0);
  __syncthreads();
}

template <class V, class X, class CT>
__global__ void __launch_bounds__(kVnecThreads)
vnec_d_kernel(int64_t m, int nL, const int* __restrict__ ptr, const V* __restrict__ val,
              const int* __restrict__ tcs, const int* __restrict__ tce, const int* __restrict__ ecr,
              const int* __restrict__ nec, const int* __restrict__ uxp, const int* __restrict__ ux,
              const int* __restrict__ vrp, const int* __restrict__ cs, const V* __restrict__ va,
              const X* __restrict__ x, X* __restrict__ y, X alpha, X beta, int* __restrict__ carry_row,
              CT* __restrict__ carry_val) {
  extern __shared__ __align__(16) unsigned char smem[];
  X* xx = reinterpret_cast<X*>(smem);
  const int t = blockIdx.x;
  stage_x(xx, ux + uxp[t], nec[t], nL, x);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int sx = tcs[2 * t], sy = tcs[2 * t + 1], ex = tce[2 * t], ey = tce[2 * t + 1];
  const int gpw = 32 / nL;  // groups per warp step
  const int k = lane % nL, gl = lane / nL;
  const uint64_t pf = policy_evict_first();
  for (int i = sx + warp; i < ex; i += nw) {
    CT acc = 0;
    for (int g = vrp[i] + gl; g < vrp[i + 1]; g += gpw)
      acc += (CT)vmul(ld_stream(va + (int64_t)g * nL + k, pf), xx[cs[g] + k]);
    acc = warp_sum(acc);
    if (lane == 0) write_row(y, i, alpha, beta, (X)acc);
  }
  if (warp == 0) {  // carry: this thread's share of row ex
    CT acc = 0;
    if (ex < m) {
      const int k0 = max(ptr[ex], sy);
      for (int q = k0 + lane; q < ey; q += 32) acc += (CT)vmul(val[q], xx[ecr[q]]);
    }
    acc = warp_sum(acc);
    if (lane == 0) {
      carry_row[t] = (ex < m) ? ex : -1;
      carry_val[t] = acc;
    }
  }
}

template <class V, class X, class CT>
__global__ void __launch_bounds__(kVnecThreads)
vnec_s_kernel(int nL, const int* __restrict__ nec, const int* __restrict__ uxp, const int* __restrict__ ux,
              const int* __restrict__ tasks, const int* __restrict__ ts, const int* __restrict__ te,
              const int* __restrict__ spv, const int* __restrict__ rb, const int* __restrict__ re,
              const int* __restrict__ rc, const V* __restrict__ rv, const X* __restrict__ x, X* __restrict__ y,
              X alpha, X beta) {
  extern __shared__ __align__(16) unsigned char smem[];
  X* xx = reinterpret_cast<X*>(smem);
  const int t = blockIdx.x;
  stage_x(xx, ux + uxp[t], nec[t], nL, x);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int T0 = ts[t], T1 = te[t], ncr = spv[t];
  const uint64_t pf = policy_evict_first();
  // cross-row groups: nL rows each, interleaved storage base + q*nL + k
  const int ngr = ncr / nL, gpw = 32 / nL;
  const int k = lane % nL, gl = lane / nL;
  for (int q0 = warp * gpw; q0 < ngr; q0 += nw * gpw) {
    const int q = q0 + gl;
    if (q < ngr) {
      const int p = T0 + q * nL;
      const int base = rb[p], rl = re[p] - rb[p];
      CT acc = 0;
      for (int c = 0; c < rl; ++c) {
        const int e = base + c * nL + k;
        acc += (CT)vmul(ld_stream(rv + e, pf), xx[rc[e]]);
      }
      write_row(y, tasks[p + k], alpha, beta, (X)acc);
    }
  }
  // in-row rows: one warp per row
  for (int p = T0 + ncr + warp; p < T1; p += nw) {
    CT acc = 0;
    for (int e = rb[p] + lane; e < re[p]; e += 32) acc += (CT)vmul(ld_stream(rv + e, pf), xx[rc[e]]);
    acc = warp_sum(acc);
    if (lane == 0) write_row(y, tasks[p], alpha, beta, (X)acc);
  }
}

// plan for the merge kernels from the structure's coordinates: pairs of
// thread_coord_start, then the last thread_coord_end
__global__ void vnec_plan_kernel(int NT, const int* __restrict__ tcs, const int* __restrict__ tce,
                                 int* __restrict__ plan) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < NT) {
    plan[2 * t] = tcs[2 * t];
    plan[2 * t + 1] = tcs[2 * t + 1];
  }
  if (t == NT - 1) {
    plan[2 * NT] = tce[2 * t];
    plan[2 * NT + 1] = tce[2 * t + 1];
  }
}

int vnec_validate(const rvvla_vnec* A, const void* x, const void* y) {
  if (!A) return fail(RVVLA_ERR_INVALID_ARG, "vnec: null descriptor");
  if (A->m < 0 || A->n < 0 || A->nz < 0 || A->NUM_THREADS_VNEC <= 0) return fail(RVVLA_ERR_INVALID_ARG, "vnec: bad sizes");
  if (A->nLanes <= 0 || A->nLanes > 32 || 32 % A->nLanes) return fail(RVVLA_ERR_FORMAT, "vnec: nLanes must divide 32");
  if (A->m > 0 && (!A->ptr || !A->thread_coord_start || !A->thread_coord_end || !y))
    return fail(RVVLA_ERR_INVALID_ARG, "vnec: null array");
  if (A->nz > 0 && (!A->indices || !A->val || !x)) return fail(RVVLA_ERR_INVALID_ARG, "vnec: null array");
  return RVVLA_OK;
}

template <class V, class X, class Ac, class P, class CT, int IPT>
int vnec_spmv_impl(const rvvla_vnec* A, X alpha, const X* x, X beta, X* y, cudaStream_t st) {
  int rc = vnec_validate(A, x, y);
  if (rc) return rc;
  if (A->m == 0) return RVVLA_OK;
  const int NT = A->NUM_THREADS_VNEC;
  const size_t xbytes = (size_t)(A->max_nec + A->nLanes) * sizeof(X);
  if (A->vnec_t == 0 || A->vnec_t == 1) {
    if (xbytes > 200 * 1024)
      return fail(RVVLA_ERR_UNSUPPORTED, "vnec: a thread's compacted x exceeds 200 KB of shared memory; build with more threads");
    if (A->vnec_t == 0) {
      Scratch sc;
      RVVLA_CUDA(sc.alloc((size_t)NT * (sizeof(int) + sizeof(CT)) + 256, st));
      int* crow = sc.as<int>();
      CT* cval = reinterpret_cast<CT*>(sc.as<char>() + ((size_t)NT * sizeof(int) + 255) / 256 * 256);
      auto k_ = vnec_d_kernel<V, X, CT>;
      if (xbytes > 48 * 1024) RVVLA_CUDA(cudaFuncSetAttribute(k_, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)xbytes));
      k_<<<NT, kVnecThreads, xbytes, st>>>(A->m, A->nLanes, A->ptr, (const V*)A->val, A->thread_coord_start,
                                           A->thread_coord_end, A->ecr_indices, A->NEC_NUM, A->use_x_ptr,
                                           A->use_x_indices, A->v_row_ptr, A->col_start, (const V*)A->val_align, x,
                                           y, alpha, beta, crow, cval);
      RVVLA_LAUNCHED("vnec_d_kernel");
      merge_fixup_kernel<X, CT><<<(NT + 255) / 256, 256, 0, st>>>(NT, (int)A->m, crow, cval, y, alpha);
      RVVLA_LAUNCHED("merge_fixup_kernel");
    } else {
      auto k_ = vnec_s_kernel<V, X, CT>;
      if (xbytes > 48 * 1024) RVVLA_CUDA(cudaFuncSetAttribute(k_, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)xbytes));
      k_<<<NT, kVnecThreads, xbytes, st>>>(A->nLanes, A->NEC_NUM, A->use_x_ptr, A->use_x_indices, A->tasks,
                                           A->task_start, A->task_end, A->spvv_len, A->row_begin, A->row_end,
                                           A->reorder_col, (const V*)A->reorder_nnz, x, y, alpha, beta);
      RVVLA_LAUNCHED("vnec_s_kernel");
    }
    return RVVLA_OK;
  }
  // L with the analysed plan: the CRS lane-run kernel on the source arrays
  if (A->plan && (A->plan_kind == 1 || A->plan_kind == 2)) {
    const rvvla_crs c{A->m, A->n, A->nz, A->ptr, A->indices, A->val, A->plan, A->plan_tiles, A->plan_kind};
    if constexpr (std::is_same<X, double>::value) return rvvla_crs_spmv_f64(&c, alpha, x, beta, y, (void*)st);
    else return rvvla_crs_spmv_f32(&c, alpha, x, beta, y, (void*)st);
  }
  // L: merge path
  const int64_t tile = (int64_t)kMergeBlock * IPT;
  const int64_t ipt = (A->nz + A->m + NT - 1) / NT;
  Scratch sc;
  int64_t ntiles;
  int32_t* plan;
  if (ipt <= tile) {
    ntiles = NT;
    RVVLA_CUDA(sc.alloc((size_t)(2 * (NT + 1)) * sizeof(int32_t) + (size_t)NT * (sizeof(int) + sizeof(CT)) + 512, st));
    plan = sc.as<int32_t>();
    vnec_plan_kernel<<<(NT + 255) / 256, 256, 0, st>>>(NT, A->thread_coord_start, A->thread_coord_end, plan);
    RVVLA_LAUNCHED("vnec_plan_kernel");
  } else {
    ntiles = crs_tiles(A->m, A->nz, IPT);
    RVVLA_CUDA(sc.alloc((size_t)(2 * (ntiles + 1)) * sizeof(int32_t) + (size_t)ntiles * (sizeof(int) + sizeof(CT)) + 512, st));
    plan = sc.as<int32_t>();
    rc = crs_plan_launch(A->m, A->nz, A->ptr, IPT, plan, st);
    if (rc) return rc;
  }
  char* after = sc.as<char>() + ((size_t)(2 * (ntiles + 1)) * sizeof(int32_t) + 255) / 256 * 256;
  int* crow = reinterpret_cast<int*>(after);
  CT* cval = reinterpret_cast<CT*>(after + ((size_t)ntiles * sizeof(int) + 255) / 256 * 256);
  prefer_shared(merge_spmv_kernel<V, X, Ac, P, CT, IPT>);
  merge_spmv_kernel<V, X, Ac, P, CT, IPT><<<(unsigned)ntiles, kMergeBlock, 0, st>>>(
      (int)A->m, (int)A->nz, A->ptr, A->indices, (const V*)A->val, x, y, alpha, beta, plan, crow, cval);
  RVVLA_LAUNCHED("merge_spmv_kernel");
  merge_fixup_kernel<X, CT><<<(unsigned)((ntiles + 255) / 256), 256, 0, st>>>((int)ntiles, (int)A->m, crow, cval, y,
                                                                              alpha);
  RVVLA_LAUNCHED("merge_fixup_kernel");
  return RVVLA_OK;
}

}  // namespace

// vnec_build.cu
template <class T>
int vnec_build_gpu(const rvvla_crs* src, int64_t NT, int force, int nL, double thr, rvvla_vnec_owned* out,
                   cudaStream_t st);

namespace {

template <class T>
int vnec_build_typed(const rvvla_crs* src, int64_t NT, int variant, rvvla_vnec_owned* out, cudaStream_t st) {
  const int64_t m = src->m, nz = src->nz;
  if (m > 0 && (!src->Rst || (nz > 0 && (!src->Col || !src->Val))))
    return fail(RVVLA_ERR_INVALID_ARG, "vnec_build: null array");
  const int nL = sizeof(T) == 4 ? 16 : 8;  // nLanes_f32 / nLanes_f64 (SpB_mxv_VNEC.h:22-23)
  const double thr = sizeof(T) == 4 ? 0.437 : 0.477;
  rvvla_vnec& h = out->h;
  h.m = m; h.n = src->n; h.nz = nz; h.NUM_THREADS_VNEC = (int32_t)NT; h.nLanes = nL;
  int rc = vnec_build_gpu<T>(src, NT, variant, nL, thr, out, st);
  if (rc) return rc;
  h.ptr = out->ptr; h.indices = out->indices; h.val = out->val;
  h.thread_coord_start = out->thread_coord_start; h.thread_coord_end = out->thread_coord_end;
  h.ecr_indices = out->ecr_indices; h.NEC_NUM = out->NEC_NUM; h.use_x_ptr = out->use_x_ptr;
  h.use_x_indices = out->use_x_indices; h.v_row_ptr = out->v_row_ptr; h.col_start = out->col_start;
  h.val_align = out->val_align; h.tasks = out->tasks; h.task_start = out->task_start; h.task_end = out->task_end;
  h.spvv_len = out->spvv_len; h.row_begin = out->row_begin; h.row_end = out->row_end;
  h.reorder_col = out->reorder_col; h.reorder_nnz = out->reorder_nnz;
  if (h.vnec_t == 2 && nz > 0) {
    // L: analyse the source CRS once for the CRS lane-run kernel
    const int dt = sizeof(T) == 8 ? RVVLA_F64 : RVVLA_F32;
    const int64_t plen = rvvla_crs_plan_len(m, nz, dt);
    RVVLA_CUDA(cudaMalloc(&out->plan, (size_t)std::max<int64_t>(plen, 1) * sizeof(int32_t)));
    const rvvla_crs c{m, src->n, nz, out->ptr, out->indices, out->val, nullptr, 0, 0};
    int64_t tiles = 0;
    int32_t kind = 0;
    if ((rc = rvvla_crs_analyze(&c, dt, out->plan, &tiles, &kind, st))) return rc;
    h.plan = out->plan; h.plan_tiles = tiles; h.plan_kind = kind;
  }
  RVVLA_CUDA(cudaStreamSynchronize(st));
  return RVVLA_OK;
}

}  // namespace
}  // namespace rvvla

using namespace rvvla;

extern "C" {

int rvvla_vnec_build(const rvvla_crs* src, int val_bytes, int64_t nthreads, int variant, rvvla_vnec_owned* out,
                     void* stream) {
  if (!src || !out) return fail(RVVLA_ERR_INVALID_ARG, "vnec_build: null argument");
  std::memset(out, 0, sizeof(*out));
  if (src->m < 0 || src->n < 0 || src->nz < 0 || (src->m > 0 && !src->Rst))
    return fail(RVVLA_ERR_INVALID_ARG, "vnec_build: bad matrix");
  if (variant < -1 || variant > 2) return fail(RVVLA_ERR_INVALID_ARG, "vnec_build: variant must be -1, 0, 1 or 2");
  const int64_t items = src->m + src->nz;
  if (nthreads <= 0) nthreads = std::max<int64_t>(1, (items + 2047) / 2048);  // one tile of merge items each
  if (nthreads > INT32_MAX) return fail(RVVLA_ERR_TOO_LARGE, "vnec_build: too many threads");
  int rc;
  if (val_bytes == 8) rc = vnec_build_typed<double>(src, nthreads, variant, out, as_stream(stream));
  else if (val_bytes == 4) rc = vnec_build_typed<float>(src, nthreads, variant, out, as_stream(stream));
  else rc = fail(RVVLA_ERR_INVALID_ARG, "vnec_build: val_bytes must be 8 or 4");
  if (rc) {
    std::string keep = rvvla_last_error();
    rvvla_vnec_free(out);
    set_error(keep);
  }
  return rc;
}

void rvvla_vnec_free(rvvla_vnec_owned* h) {
  if (!h) return;
  void* ptrs[] = {h->ptr, h->indices, h->val, h->thread_coord_start, h->thread_coord_end, h->ecr_indices, h->NEC_NUM,
                  h->use_x_ptr, h->use_x_indices, h->v_row_ptr, h->col_start, h->val_align, h->tasks, h->task_start,
                  h->task_end, h->spvv_len, h->row_begin, h->row_end, h->reorder_col, h->reorder_nnz, h->plan};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  std::memset(h, 0, sizeof(*h));
}

int rvvla_vnec_spmv_f64(const rvvla_vnec* A, double alpha, const double* x, double beta, double* y, void* stream) {
  return vnec_spmv_impl<double, double, double, double, double, MergeCfg<double>::IPT>(A, alpha, x, beta, y,
                                                                                      as_stream(stream));
}

int rvvla_vnec_spmv_f32(const rvvla_vnec* A, float alpha, const float* x, float beta, float* y, void* stream) {
  return vnec_spmv_impl<float, float, float, float, float, MergeCfg<float>::IPT>(A, alpha, x, beta, y,
                                                                               as_stream(stream));
}

}  // extern "C"
