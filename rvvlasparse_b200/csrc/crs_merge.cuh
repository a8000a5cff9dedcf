// crs_merge.cuh — merge-path CSR kernels (plan, tile SpMV, carry fix-up),
// shared by crs.cu (spMtxCRS) and vnec.cu (spMtxVNEC, variant L).
#pragma once
#include "rvvla_internal.cuh"

namespace rvvla {

constexpr int kMergeBlock = 256;

template <class V> struct MergeCfg;
template <> struct MergeCfg<double> { static constexpr int IPT = 8; };
template <> struct MergeCfg<float> { static constexpr int IPT = 12; };
template <> struct MergeCfg<__nv_bfloat16> { static constexpr int IPT = 12; };

// ---- accumulator operations (double, float, compensated fp32)
__device__ __forceinline__ void acc_zero(double& a) { a = 0.0; }
__device__ __forceinline__ void acc_zero(float& a) { a = 0.f; }
__device__ __forceinline__ void acc_zero(CompF32& a) { a.s = 0.f; a.c = 0.f; }
__device__ __forceinline__ void acc_add(double& a, double p) { a += p; }
__device__ __forceinline__ void acc_add(float& a, float p) { a += p; }
__device__ __forceinline__ void acc_add(CompF32& a, float p) { a.add(p); }
__device__ __forceinline__ void acc_merge(double& a, const double& b) { a += b; }
__device__ __forceinline__ void acc_merge(float& a, const float& b) { a += b; }
__device__ __forceinline__ void acc_merge(CompF32& a, const CompF32& b) { a.add(b); }
__device__ __forceinline__ double acc_shfl_up(double a, int d) { return __shfl_up_sync(0xffffffffu, a, d); }
__device__ __forceinline__ float acc_shfl_up(float a, int d) { return __shfl_up_sync(0xffffffffu, a, d); }
__device__ __forceinline__ CompF32 acc_shfl_up(CompF32 a, int d) {
  CompF32 r;
  r.s = __shfl_up_sync(0xffffffffu, a.s, d);
  r.c = __shfl_up_sync(0xffffffffu, a.c, d);
  return r;
}
__device__ __forceinline__ double acc_shfl_xor(double a, int d) { return __shfl_xor_sync(0xffffffffu, a, d); }
__device__ __forceinline__ float acc_shfl_xor(float a, int d) { return __shfl_xor_sync(0xffffffffu, a, d); }
__device__ __forceinline__ CompF32 acc_shfl_xor(CompF32 a, int d) {
  CompF32 r;
  r.s = __shfl_xor_sync(0xffffffffu, a.s, d);
  r.c = __shfl_xor_sync(0xffffffffu, a.c, d);
  return r;
}
__device__ __forceinline__ double acc_bcast(double a, int l) { return __shfl_sync(0xffffffffu, a, l); }
__device__ __forceinline__ float acc_bcast(float a, int l) { return __shfl_sync(0xffffffffu, a, l); }
__device__ __forceinline__ CompF32 acc_bcast(CompF32 a, int l) {
  CompF32 r;
  r.s = __shfl_sync(0xffffffffu, a.s, l);
  r.c = __shfl_sync(0xffffffffu, a.c, l);
  return r;
}
__device__ __forceinline__ double acc_out(double a) { return a; }
__device__ __forceinline__ float acc_out(float a) { return a; }
__device__ __forceinline__ float acc_out(const CompF32& a) { return a.value(); }
__device__ __forceinline__ double acc_carry(double a) { return a; }
__device__ __forceinline__ float acc_carry(float a) { return a; }
__device__ __forceinline__ double acc_carry(const CompF32& a) { return (double)a.s + (double)a.c; }

template <class V, class X>
__device__ __forceinline__ auto vmul(V v, X x) { return v * x; }
template <>
__device__ __forceinline__ auto vmul<__nv_bfloat16, float>(__nv_bfloat16 v, float x) { return __bfloat162float(v) * x; }

// Merge-path split points for tile boundaries t*tile_items, t = 0..ntiles:
// plan[2t] = rows whose end precedes the boundary, plan[2t+1] = nonzeros
// before it.  Same search as MergePathDivide (src/rvv/spmv_mtx_vnec.cpp:42-71)
// with list A = row ends (Rst+1) and list B = 0..nnz-1.
__global__ void merge_plan_kernel(int m, int nnz, const int* __restrict__ Rst, int tile_items, int ntiles,
                                  int* __restrict__ plan);

template <class X>
__device__ __forceinline__ void write_row(X* y, int r, X alpha, X beta, X o) {
  if (beta == X(0)) y[r] = alpha * o;
  else y[r] = alpha * o + beta * y[r];
}

// One CTA per tile of kMergeBlock*IPT merge items.
template <class V, class X, class Ac, class P, class CT, int IPT>
__global__ void __launch_bounds__(kMergeBlock)
merge_spmv_kernel(int m, int nnz, const int* __restrict__ Rst, const int* __restrict__ Col,
                  const V* __restrict__ Val, const X* __restrict__ x, X* __restrict__ y, X alpha, X beta,
                  const int* __restrict__ plan, int* __restrict__ carry_row, CT* __restrict__ carry_val) {
  constexpr int TILE = kMergeBlock * IPT;
  constexpr int NW = kMergeBlock / 32;
  // rows + nonzeros of a tile add up to TILE, so row ends (int) and products
  // share one buffer: row ends from the front, products after them.
  __shared__ __align__(16) unsigned char s_buf[TILE * (sizeof(P) > sizeof(int) ? sizeof(P) : sizeof(int)) + 16];
  __shared__ Ac s_scan[kMergeBlock];
  __shared__ int s_key[kMergeBlock];
  __shared__ int s_wk0[NW], s_wk31[NW];
  __shared__ Ac s_wv[NW];

  const int t = blockIdx.x, tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int x0 = plan[2 * t], y0 = plan[2 * t + 1];
  const int nrows = plan[2 * t + 2] - x0, nnzt = plan[2 * t + 3] - y0;
  int* s_rowend = reinterpret_cast<int*>(s_buf);
  P* s_prod = reinterpret_cast<P*>(s_buf + (((size_t)nrows * sizeof(int) + sizeof(P) - 1) / sizeof(P)) * sizeof(P));
  const uint64_t pf = policy_evict_first(), pl = policy_evict_last();

  // 1. stage row ends and products
  for (int i = tid; i < nrows; i += kMergeBlock) s_rowend[i] = ld_stream(Rst + x0 + 1 + i, pf);
  {
    int cidx[IPT];
    V vv[IPT];
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
      const int j = tid + k * kMergeBlock;
      if (j < nnzt) {
        cidx[k] = ld_stream(Col + y0 + j, pf);
        vv[k] = ld_stream(Val + y0 + j, pf);
      }
    }
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
      const int j = tid + k * kMergeBlock;
      if (j < nnzt) s_prod[j] = vmul(vv[k], ld_keep(x + cidx[k], pl));
    }
  }
  __syncthreads();

  // 2. this thread's merge-path start inside the tile
  const int items = nrows + nnzt;
  const int diag = min(tid * IPT, items);
  int lo = max(diag - nnzt, 0), hi = min(diag, nrows);
  while (lo < hi) {
    const int piv = (lo + hi) >> 1;
    if (s_rowend[piv] <= y0 + diag - piv - 1) lo = piv + 1;
    else hi = piv;
  }
  int xi = lo, yi = diag - lo;
  const int cnt = min(diag + IPT, items) - diag;
  Ac run, first;
  acc_zero(run);
  acc_zero(first);
  int first_row = -1;
#pragma unroll
  for (int k = 0; k < IPT; ++k) {
    if (k < cnt) {
      if (xi < nrows && (yi >= nnzt || s_rowend[xi] <= y0 + yi)) {
        if (first_row < 0) { first_row = xi; first = run; }
        else write_row(y, x0 + xi, alpha, beta, (X)acc_out(run));
        acc_zero(run);
        ++xi;
      } else {
        acc_add(run, s_prod[yi]);
        ++yi;
      }
    }
  }

  // 3. block-wide segmented scan of (row in progress, partial) over threads
  int key = xi;
  Ac v = run;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    Ac ov = acc_shfl_up(v, d);
    int ok = __shfl_up_sync(0xffffffffu, key, d);
    if (lane >= d && ok == key) acc_merge(v, ov);
  }
  if (lane == 31) { s_wk31[warp] = key; s_wv[warp] = v; }
  if (lane == 0) s_wk0[warp] = key;
  __syncthreads();
  const int k0 = __shfl_sync(0xffffffffu, key, 0);
  if (k0 == key) {
    for (int w2 = warp - 1; w2 >= 0; --w2) {
      if (s_wk31[w2] != key) break;
      acc_merge(v, s_wv[w2]);
      if (s_wk0[w2] != key) break;
    }
  }
  s_scan[tid] = v;
  s_key[tid] = key;
  __syncthreads();
  if (first_row >= 0) {
    Ac tot = first;
    if (tid > 0 && s_key[tid - 1] == first_row) acc_merge(tot, s_scan[tid - 1]);
    write_row(y, x0 + first_row, alpha, beta, (X)acc_out(tot));
  }
  // 4. carry of the row that continues into the next tile
  if (tid == kMergeBlock - 1) {
    const int r = x0 + s_key[tid];
    carry_row[t] = (r < m) ? r : -1;
    carry_val[t] = acc_carry(s_scan[tid]);
  }
}

// Adds tile carries in tile order; a run of tiles carrying into one row is
// summed first (in fp64 for the mixed forms) and added once.
template <class X, class CT>
__global__ void merge_fixup_kernel(int ntiles, int m, const int* __restrict__ carry_row,
                                   const CT* __restrict__ carry_val, X* __restrict__ y, X alpha) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntiles) return;
  const int r = carry_row[t];
  if (r < 0 || r >= m) return;
  if (t > 0 && carry_row[t - 1] == r) return;
  CT s = carry_val[t];
  for (int u = t + 1; u < ntiles && carry_row[u] == r; ++u) s += carry_val[u];
  y[r] += alpha * (X)s;
}

int64_t crs_tiles(int64_t m, int64_t nz, int ipt);
int crs_validate(const rvvla_crs* A, const void* x, const void* y);
int crs_plan_launch(int64_t m, int64_t nz, const int32_t* Rst, int ipt, int32_t* plan, cudaStream_t st);

}  // namespace rvvla
