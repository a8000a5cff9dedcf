// sell.cu — spMtxSELL_C_Sigma on sm_100a: GPU builder and the SpMV stages.
//
// Layout (include/SELL_C_Sigma.h:23-40 of the reference) as read by
// src/scalar/spmv_mtx_sell_c_sigma.cpp:52-98: slice s holds sorted rows
// [vSBs[s], vSBs[s]+vBs[s]), width vCl[s], element (k, j) at
// vCs[s] + j*vBs[s] + k; vPerm[sorted] = original row.  The reference ships
// no builder; rows are sorted by length (descending, stable) inside windows
// of Sigma rows, slices of C rows, padding value 0 / column 0 — the same
// layout as the oracle's builder, bit for bit.
//
// SpMV: one thread per sorted row.  With C = 32 a warp is a slice: every
// column step j is one coalesced 32-wide load of values and columns (L2
// evict-first) plus an x gather (evict-last).  Stages follow the reference:
// PREPARATION y := y[perm], MULT in permuted space (:52-98), GET_RESULTS
// y[perm] := y (:100-127); ALL fuses them by reading and writing y through
// vPerm, as the RVV kernel does (src/rvv/spmv_mtx_sell_c_sigma.cpp:78-83).
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cstring>
#include <string>

#include "crs_merge.cuh"
#include "rvvla_internal.cuh"
#include "scan.cuh"

namespace rvvla {
namespace {

// key = (window << 32) | (0xFFFFFFFF - length): ascending key order is
// window-major, length descending; the radix sort is stable, so equal
// lengths keep source order.
__global__ void sell_keys_kernel(int64_t m, int64_t sigma, const int* __restrict__ Rst, uint64_t* __restrict__ key,
                                 uint32_t* __restrict__ idx) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const uint32_t len = (uint32_t)(Rst[i + 1] - Rst[i]);
  key[i] = ((uint64_t)(i / sigma) << 32) | (uint64_t)(0xFFFFFFFFu - len);
  idx[i] = (uint32_t)i;
}

__global__ void sell_slices_kernel(int64_t m, int64_t C, int64_t cnt_b, const int* __restrict__ Rst,
                                   const uint32_t* __restrict__ perm, int* __restrict__ vCl, int* __restrict__ vBs,
                                   int* __restrict__ vSBs, int64_t* __restrict__ area) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= cnt_b) return;
  const int64_t r0 = s * C, r1 = min(m, r0 + C);
  int w = 0;
  for (int64_t r = r0; r < r1; ++r) {
    const uint32_t row = perm[r];
    w = max(w, Rst[row + 1] - Rst[row]);
  }
  vCl[s] = w;
  vBs[s] = (int)(r1 - r0);
  vSBs[s] = (int)r0;
  area[s] = (int64_t)w * (r1 - r0);
}

__global__ void sell_cs_kernel(int64_t cnt_b, const int64_t* __restrict__ off, int* __restrict__ vCs) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s < cnt_b) vCs[s] = (int)off[s];
}

template <int VB>
__global__ void sell_fill_kernel(int64_t m, int64_t C, const int* __restrict__ Rst, const int* __restrict__ Col,
                                 const uint8_t* __restrict__ Val, const uint32_t* __restrict__ perm,
                                 const int* __restrict__ vCl, const int* __restrict__ vCs,
                                 const int* __restrict__ vBs, uint32_t* __restrict__ vCol,
                                 uint8_t* __restrict__ vVal) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= m) return;
  const int64_t s = g / C, k = g - s * C;
  const uint32_t row = perm[g];
  const int kb = Rst[row], len = Rst[row + 1] - kb;
  const int w = vCl[s], bs = vBs[s];
  int64_t p = vCs[s] + k;
  for (int j = 0; j < w; ++j, p += bs) {
    if (j < len) {
      vCol[p] = (uint32_t)Col[kb + j];
#pragma unroll
      for (int q = 0; q < VB; ++q) vVal[p * VB + q] = Val[(int64_t)(kb + j) * VB + q];
    } else {
      vCol[p] = 0u;
#pragma unroll
      for (int q = 0; q < VB; ++q) vVal[p * VB + q] = 0;
    }
  }
}

// MODE 0: MULT (permuted y), 1: ALL (y through vPerm)
template <class V, class X, class Ac, int MODE>
__global__ void __launch_bounds__(256)
sell_spmv_kernel(int64_t m, int64_t C, const int* __restrict__ vCl, const int* __restrict__ vCs,
                 const int* __restrict__ vBs, const int* __restrict__ vSBs, const uint32_t* __restrict__ vCol,
                 const uint32_t* __restrict__ vPerm, const V* __restrict__ vVal, const X* __restrict__ x,
                 X* __restrict__ y, X alpha, X beta) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= m) return;
  const int64_t s = g / C;
  const int64_t k = g - s * C;
  const int w = vCl[s], bs = vBs[s];
  const uint64_t pf = policy_evict_first(), pl = policy_evict_last();
  const int64_t base = vCs[s] + k;
  Ac acc;
  acc_zero(acc);
  int j = 0;
  for (; j + 4 <= w; j += 4) {
    uint32_t c[4];
    V v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      c[u] = ld_stream(vCol + base + (int64_t)(j + u) * bs, pf);
      v[u] = ld_stream(vVal + base + (int64_t)(j + u) * bs, pf);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) acc_add(acc, vmul(v[u], ld_keep(x + c[u], pl)));
  }
  for (; j < w; ++j) {
    const uint32_t c = ld_stream(vCol + base + (int64_t)j * bs, pf);
    acc_add(acc, vmul(ld_stream(vVal + base + (int64_t)j * bs, pf), ld_keep(x + c, pl)));
  }
  const int64_t out = (MODE == 1) ? (int64_t)vPerm[vSBs[s] + k] : (int64_t)vSBs[s] + k;
  write_row(y, (int)out, alpha, beta, (X)acc_out(acc));
}

// C == 32: a warp per slice (lane = row of the slice, column-major loads are
// coalesced).  A CTA covers 8 consecutive slices; slices wider than
// kSellWide columns (the long rows that sigma-sorting gathers at the head of
// a window) are shared by all 8 warps of the CTA, each taking every eighth
// group of 4 columns, and the 8 partial sums of a row are merged in warp
// order through shared memory, so a wide slice costs the CTA width/8 steps
// instead of holding one warp for width steps.
constexpr int kSellWide = 64;

template <class V, class X, class Ac, int MODE>
__global__ void __launch_bounds__(256)
sell_warp_kernel(int64_t cnt_b, const int* __restrict__ vCl, const int* __restrict__ vCs,
                 const int* __restrict__ vBs, const int* __restrict__ vSBs, const uint32_t* __restrict__ vCol,
                 const uint32_t* __restrict__ vPerm, const V* __restrict__ vVal, const X* __restrict__ x,
                 X* __restrict__ y, X alpha, X beta) {
  __shared__ Ac red[8][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t s0 = (int64_t)blockIdx.x * 8;
  const uint64_t pf = policy_evict_first(), pl = policy_evict_last();
  {
    const int64_t s = s0 + warp;
    if (s < cnt_b) {
      const int w = vCl[s], bs = vBs[s];
      if (w <= kSellWide && lane < bs) {
        const int64_t base = vCs[s] + lane;
        Ac acc;
        acc_zero(acc);
        // columns in flight: 4 for 8-byte values, 8 for narrower ones
        constexpr int U = sizeof(V) >= 8 ? 4 : 8;
        int j = 0;
        for (; j + U <= w; j += U) {
          uint32_t c[U];
          V v[U];
#pragma unroll
          for (int u = 0; u < U; ++u) {
            c[u] = ld_stream(vCol + base + (int64_t)(j + u) * bs, pf);
            v[u] = ld_stream(vVal + base + (int64_t)(j + u) * bs, pf);
          }
#pragma unroll
          for (int u = 0; u < U; ++u) acc_add(acc, vmul(v[u], ld_keep(x + c[u], pl)));
        }
        for (; j < w; ++j) {
          const uint32_t c = ld_stream(vCol + base + (int64_t)j * bs, pf);
          acc_add(acc, vmul(ld_stream(vVal + base + (int64_t)j * bs, pf), ld_keep(x + c, pl)));
        }
        const int64_t out = (MODE == 1) ? (int64_t)vPerm[vSBs[s] + lane] : (int64_t)vSBs[s] + lane;
        write_row(y, (int)out, alpha, beta, (X)acc_out(acc));
      }
    }
  }
  for (int q = 0; q < 8; ++q) {  // wide slices: the whole CTA (uniform branches)
    const int64_t s = s0 + q;
    if (s >= cnt_b) break;
    const int w = vCl[s];
    if (w <= kSellWide) continue;
    const int bs = vBs[s];
    Ac acc;
    acc_zero(acc);
    if (lane < bs) {
      const int64_t base = vCs[s] + lane;
      for (int j0 = warp * 4; j0 < w; j0 += 32) {
        uint32_t c[4];
        V v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const bool in = j0 + u < w;
          c[u] = in ? ld_stream(vCol + base + (int64_t)(j0 + u) * bs, pf) : 0u;
          v[u] = in ? ld_stream(vVal + base + (int64_t)(j0 + u) * bs, pf) : V(0.0f);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
          if (j0 + u < w) acc_add(acc, vmul(v[u], ld_keep(x + c[u], pl)));
      }
    }
    red[warp][lane] = acc;
    __syncthreads();
    if (warp == 0 && lane < bs) {
      Ac t = red[0][lane];
#pragma unroll
      for (int k = 1; k < 8; ++k) acc_merge(t, red[k][lane]);
      const int64_t out = (MODE == 1) ? (int64_t)vPerm[vSBs[s] + lane] : (int64_t)vSBs[s] + lane;
      write_row(y, (int)out, alpha, beta, (X)acc_out(t));
    }
    __syncthreads();
  }
}

template <class X>
__global__ void sell_permute_kernel(int64_t m, const uint32_t* __restrict__ perm, const X* __restrict__ src,
                                    X* __restrict__ dst, int gather) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  if (gather) dst[i] = src[perm[i]];  // PREPARATION: y[i] = y_old[perm[i]]
  else dst[perm[i]] = src[i];         // GET_RESULTS: y[perm[i]] = y_old[i]
}

int sell_validate(const rvvla_sell* A, const void* x, const void* y) {
  if (!A) return fail(RVVLA_ERR_INVALID_ARG, "sell: null descriptor");
  if (A->m < 0 || A->n < 0 || A->cnt_b < 0 || A->C <= 0) return fail(RVVLA_ERR_INVALID_ARG, "sell: bad sizes");
  if (A->cnt_b != (A->m + A->C - 1) / A->C)
    return fail(RVVLA_ERR_FORMAT, "sell: the sm_100a kernel needs slices of C rows (cnt_b = ceil(m/C))");
  if (A->m > 0 && (!A->vCl || !A->vCs || !A->vBs || !A->vSBs || !A->vPerm || !y))
    return fail(RVVLA_ERR_INVALID_ARG, "sell: null array");
  if (A->len > 0 && (!A->vCol || !A->vVal || !x)) return fail(RVVLA_ERR_INVALID_ARG, "sell: null array");
  return RVVLA_OK;
}

template <class V, class X, class Ac>
int sell_spmv_impl(const rvvla_sell* A, int stage, X alpha, const X* x, X beta, X* y, cudaStream_t st) {
  int rc = sell_validate(A, x, y);
  if (rc) return rc;
  if (A->m == 0) return RVVLA_OK;
  const unsigned blocks = (unsigned)((A->m + 255) / 256);
  if (stage == RVVLA_STAGE_PREPARATION || stage == RVVLA_STAGE_GET_RESULTS) {
    Scratch sc;
    RVVLA_CUDA(sc.alloc((size_t)A->m * sizeof(X), st));
    RVVLA_CUDA(cudaMemcpyAsync(sc.p, y, (size_t)A->m * sizeof(X), cudaMemcpyDeviceToDevice, st));
    sell_permute_kernel<X><<<blocks, 256, 0, st>>>(A->m, A->vPerm, sc.as<X>(), y,
                                                   stage == RVVLA_STAGE_PREPARATION ? 1 : 0);
    RVVLA_LAUNCHED("sell_permute_kernel");
    return RVVLA_OK;
  }
  const V* vv = (const V*)A->vVal;
  if (A->C == 32 && (stage == RVVLA_STAGE_MULT || stage == RVVLA_STAGE_ALL)) {
    const unsigned wblocks = (unsigned)((A->cnt_b + 7) / 8);
    if (stage == RVVLA_STAGE_MULT)
      sell_warp_kernel<V, X, Ac, 0><<<wblocks, 256, 0, st>>>(A->cnt_b, A->vCl, A->vCs, A->vBs, A->vSBs, A->vCol,
                                                             A->vPerm, vv, x, y, alpha, beta);
    else
      sell_warp_kernel<V, X, Ac, 1><<<wblocks, 256, 0, st>>>(A->cnt_b, A->vCl, A->vCs, A->vBs, A->vSBs, A->vCol,
                                                             A->vPerm, vv, x, y, alpha, beta);
    RVVLA_LAUNCHED("sell_warp_kernel");
    return RVVLA_OK;
  }
  if (stage == RVVLA_STAGE_MULT)
    sell_spmv_kernel<V, X, Ac, 0><<<blocks, 256, 0, st>>>(A->m, A->C, A->vCl, A->vCs, A->vBs, A->vSBs, A->vCol,
                                                          A->vPerm, vv, x, y, alpha, beta);
  else if (stage == RVVLA_STAGE_ALL)
    sell_spmv_kernel<V, X, Ac, 1><<<blocks, 256, 0, st>>>(A->m, A->C, A->vCl, A->vCs, A->vBs, A->vSBs, A->vCol,
                                                          A->vPerm, vv, x, y, alpha, beta);
  else
    return fail(RVVLA_ERR_INVALID_ARG, "sell: unknown stage");
  RVVLA_LAUNCHED("sell_spmv_kernel");
  return RVVLA_OK;
}

}  // namespace

int sell_build_impl(const rvvla_crs* src, int vb, int64_t C, int64_t sigma, rvvla_sell_owned* out, cudaStream_t st) {
  if (!src || !out) return fail(RVVLA_ERR_INVALID_ARG, "sell_build: null argument");
  std::memset(out, 0, sizeof(*out));
  if (C <= 0) return fail(RVVLA_ERR_INVALID_ARG, "SELL: C must be positive");
  if (vb != 8 && vb != 4 && vb != 2) return fail(RVVLA_ERR_INVALID_ARG, "sell_build: val_bytes must be 8, 4 or 2");
  if (sigma <= 0) sigma = 1;
  const int64_t m = src->m;
  if (m < 0 || src->n < 0 || src->nz < 0) return fail(RVVLA_ERR_INVALID_ARG, "sell_build: bad sizes");
  if (m >= INT32_MAX) return fail(RVVLA_ERR_TOO_LARGE, "sell_build: m beyond int32");
  const int64_t cnt_b = (m + C - 1) / C;
  rvvla_sell& h = out->h;
  h.m = m; h.n = src->n; h.nz = src->nz; h.cnt_b = cnt_b; h.C = (int32_t)C; h.Sigma = (int32_t)sigma;
  RVVLA_CUDA(cudaMalloc(&out->vPerm, (size_t)std::max<int64_t>(m, 1) * sizeof(uint32_t)));
  RVVLA_CUDA(cudaMalloc(&out->vCl, (size_t)std::max<int64_t>(cnt_b, 1) * sizeof(int32_t)));
  RVVLA_CUDA(cudaMalloc(&out->vCs, (size_t)std::max<int64_t>(cnt_b, 1) * sizeof(int32_t)));
  RVVLA_CUDA(cudaMalloc(&out->vBs, (size_t)std::max<int64_t>(cnt_b, 1) * sizeof(int32_t)));
  RVVLA_CUDA(cudaMalloc(&out->vSBs, (size_t)std::max<int64_t>(cnt_b, 1) * sizeof(int32_t)));
  int64_t total = 0;
  if (m > 0) {
    Scratch s_key, s_key2, s_idx, s_tmp, s_area, s_off;
    RVVLA_CUDA(s_key.alloc((size_t)m * sizeof(uint64_t), st));
    RVVLA_CUDA(s_key2.alloc((size_t)m * sizeof(uint64_t), st));
    RVVLA_CUDA(s_idx.alloc((size_t)m * sizeof(uint32_t), st));
    sell_keys_kernel<<<(unsigned)((m + 255) / 256), 256, 0, st>>>(m, sigma, src->Rst, s_key.as<uint64_t>(),
                                                                   s_idx.as<uint32_t>());
    RVVLA_LAUNCHED("sell_keys_kernel");
    int end_bit = 32;
    for (int64_t w = (m + sigma - 1) / sigma; w > 1; w >>= 1) end_bit++;
    end_bit = std::min(64, end_bit + 1);
    size_t tmp_bytes = 0;
    RVVLA_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, s_key.as<uint64_t>(), s_key2.as<uint64_t>(),
                                               s_idx.as<uint32_t>(), out->vPerm, (int)m, 0, end_bit, st));
    RVVLA_CUDA(s_tmp.alloc(tmp_bytes, st));
    RVVLA_CUDA(cub::DeviceRadixSort::SortPairs(s_tmp.p, tmp_bytes, s_key.as<uint64_t>(), s_key2.as<uint64_t>(),
                                               s_idx.as<uint32_t>(), out->vPerm, (int)m, 0, end_bit, st));
    count_launch(3);
    RVVLA_CUDA(s_area.alloc((size_t)(cnt_b + 1) * sizeof(int64_t), st));
    RVVLA_CUDA(s_off.alloc((size_t)(cnt_b + 1) * sizeof(int64_t), st));
    sell_slices_kernel<<<(unsigned)((cnt_b + 255) / 256), 256, 0, st>>>(m, C, cnt_b, src->Rst, out->vPerm, out->vCl,
                                                                         out->vBs, out->vSBs, s_area.as<int64_t>());
    RVVLA_LAUNCHED("sell_slices_kernel");
    int rc = exclusive_scan_i64(s_area.as<int64_t>(), s_off.as<int64_t>(), cnt_b, st);
    if (rc) return rc;
    RVVLA_CUDA(cudaMemcpyAsync(&total, s_off.as<int64_t>() + cnt_b, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    RVVLA_CUDA(cudaStreamSynchronize(st));
    if (total > INT32_MAX) return fail(RVVLA_ERR_TOO_LARGE, "SELL: padded size exceeds int32 offsets");
    sell_cs_kernel<<<(unsigned)((cnt_b + 255) / 256), 256, 0, st>>>(cnt_b, s_off.as<int64_t>(), out->vCs);
    RVVLA_LAUNCHED("sell_cs_kernel");
    RVVLA_CUDA(cudaMalloc(&out->vCol, (size_t)std::max<int64_t>(total, 1) * sizeof(uint32_t)));
    RVVLA_CUDA(cudaMalloc(&out->vVal, (size_t)std::max<int64_t>(total, 1) * vb));
    const unsigned blocks = (unsigned)((m + 255) / 256);
    if (vb == 8) sell_fill_kernel<8><<<blocks, 256, 0, st>>>(m, C, src->Rst, src->Col, (const uint8_t*)src->Val, out->vPerm, out->vCl, out->vCs, out->vBs, out->vCol, (uint8_t*)out->vVal);
    else if (vb == 4) sell_fill_kernel<4><<<blocks, 256, 0, st>>>(m, C, src->Rst, src->Col, (const uint8_t*)src->Val, out->vPerm, out->vCl, out->vCs, out->vBs, out->vCol, (uint8_t*)out->vVal);
    else sell_fill_kernel<2><<<blocks, 256, 0, st>>>(m, C, src->Rst, src->Col, (const uint8_t*)src->Val, out->vPerm, out->vCl, out->vCs, out->vBs, out->vCol, (uint8_t*)out->vVal);
    RVVLA_LAUNCHED("sell_fill_kernel");
  } else {
    RVVLA_CUDA(cudaMalloc(&out->vCol, sizeof(uint32_t)));
    RVVLA_CUDA(cudaMalloc(&out->vVal, 8));
  }
  h.len = total;
  h.vCl = out->vCl; h.vCs = out->vCs; h.vBs = out->vBs; h.vSBs = out->vSBs;
  h.vCol = out->vCol; h.vPerm = out->vPerm; h.vVal = out->vVal;
  RVVLA_CUDA(cudaStreamSynchronize(st));
  return RVVLA_OK;
}

}  // namespace rvvla

using namespace rvvla;

extern "C" {

int rvvla_sell_build(const rvvla_crs* src, int val_bytes, int64_t C, int64_t sigma, rvvla_sell_owned* out,
                     void* stream) {
  int rc = sell_build_impl(src, val_bytes, C, sigma, out, as_stream(stream));
  if (rc && out) {
    std::string keep = rvvla_last_error();
    rvvla_sell_free(out);
    set_error(keep);
  }
  return rc;
}

void rvvla_sell_free(rvvla_sell_owned* h) {
  if (!h) return;
  cudaFree(h->vCl);
  cudaFree(h->vCs);
  cudaFree(h->vBs);
  cudaFree(h->vSBs);
  cudaFree(h->vCol);
  cudaFree(h->vPerm);
  cudaFree(h->vVal);
  std::memset(h, 0, sizeof(*h));
}

int rvvla_sell_spmv_f64(const rvvla_sell* A, int stage, double alpha, const double* x, double beta, double* y,
                        void* stream) {
  return sell_spmv_impl<double, double, double>(A, stage, alpha, x, beta, y, as_stream(stream));
}

int rvvla_sell_spmv_f32(const rvvla_sell* A, int stage, float alpha, const float* x, float beta, float* y,
                        void* stream) {
  return sell_spmv_impl<float, float, float>(A, stage, alpha, x, beta, y, as_stream(stream));
}

int rvvla_sell_spmv_mixed(const rvvla_sell* A, int val_type, float alpha, const float* x, float beta, float* y,
                          void* stream) {
  if (val_type == RVVLA_F32)
    return sell_spmv_impl<float, float, CompF32>(A, RVVLA_STAGE_ALL, alpha, x, beta, y, as_stream(stream));
  if (val_type == RVVLA_BF16)
    return sell_spmv_impl<__nv_bfloat16, float, CompF32>(A, RVVLA_STAGE_ALL, alpha, x, beta, y, as_stream(stream));
  return fail(RVVLA_ERR_INVALID_ARG, "sell_spmv_mixed: val_type must be RVVLA_F32 or RVVLA_BF16");
}

}  // extern "C"
