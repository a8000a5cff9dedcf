// lav.cu — spMtxLAV on sm_100a: SpMV (the builder is in lav_build.cu, on the GPU).
//
// Layout (include/LAV.h:10-31 of the reference) as read by
// src/scalar/spmv_mtx_lav.cpp:36-79: dense columns cut into segments; per
// segment, chunks of SIMD_Lanes rows (out_order), each chunk a run of steps
// (chunk_offsets, relative to segment_ptr[s]); steps before
// chunk_offsets_full_mask use every lane, later ones mask[step] lanes (a
// prefix); val/col_id lane-major per step; the remaining entries in
// sparse_part (CRS, which applies beta to every row).  The reference ships no
// builder; this one reproduces the oracle's: dense columns = the densest
// columns holding >= (1-T) of the nonzeros, segments of segment_len columns
// in density order, one global row chunking (rows by dense count,
// descending) with each segment ordering a chunk's rows by their count in
// that segment.
//
// SpMV: sparse part through the CRS kernels (with its analysis plan), then
// one launch per segment (the reference's segment loop, :147-174): a thread
// per (chunk, lane) sums its steps and adds alpha*sum to y[out_order]; a row
// appears once per segment, so the launches need no atomics.
#include <algorithm>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "crs_merge.cuh"
#include "rvvla_internal.cuh"

extern "C" int rvvla_crs_spmv_f64(const rvvla_crs*, double, const double*, double, double*, void*);
extern "C" int rvvla_crs_spmv_f32(const rvvla_crs*, float, const float*, float, float*, void*);

namespace rvvla {
namespace {

template <class V, class X, class CT>
__global__ void __launch_bounds__(256)
lav_segment_kernel(int64_t s, int64_t L, int64_t cc, const int* __restrict__ co, const int* __restrict__ cf,
                   const uint64_t* __restrict__ sp, const uint32_t* __restrict__ oo, const uint16_t* __restrict__ mk,
                   const V* __restrict__ val, const uint32_t* __restrict__ col, const X* __restrict__ x,
                   X* __restrict__ y, X alpha) {
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= cc * L) return;
  const int64_t c = gid / L, i = gid - c * L;
  const int64_t sh = (cc + 1) * s;
  const int st = co[sh + c], en = co[sh + c + 1], fe = cf[s * cc + c];
  if (st >= en) return;
  const int64_t base = (int64_t)sp[s];
  const bool active = (fe > st) || (i < (int64_t)mk[base + st]);
  if (!active) return;
  const uint64_t pf = policy_evict_first(), pl = policy_evict_last();
  CT acc = 0;
  for (int q = st; q < fe; ++q) {
    const int64_t e = (base + q) * L + i;
    acc += (CT)vmul(ld_stream(val + e, pf), ld_keep(x + ld_stream(col + e, pf), pl));
  }
  for (int q = fe; q < en; ++q) {
    if (i >= (int64_t)mk[base + q]) break;  // masks are non-increasing
    const int64_t e = (base + q) * L + i;
    acc += (CT)vmul(ld_stream(val + e, pf), ld_keep(x + ld_stream(col + e, pf), pl));
  }
  const uint32_t r = oo[(c + cc * s) * L + i];
  y[r] += alpha * (X)acc;
}

// All segments in one pass (L divides 32).  Blocks [0, nlong) take the
// long chunks [0, nlong), one CTA each: thread (g, i) sums every G-th step
// (G = 256 / L) of lane i, the groups' partial sums are added in group
// order through shared memory, and thread j < L owns slot j.  The remaining
// blocks give lane (c, j) of a warp slot j of chunk c >= nlong, i.e. row
// row_order[c*L + j]: in every segment lane (c, i) sums its steps for the row
// the segment placed at lane i, and the slot owner takes that sum from lane
// lane_of_slot[(s, c, j)] with a shuffle.  Either way a row's segment sums
// are added in segment order and y is read-modified-written once (after the
// sparse part has applied beta).  Chunks are cut from rows sorted by dense
// count, so the long chunks lead and their CTAs start first.
//
// Loads: each thread issues all loads of kLavU steps before using any (steps
// past the chunk's end are clamped to its last step, which holds L slots,
// and dropped); x is gathered at min(col, n-1) so that padding slots need
// no mask test first, and a product counts only where the step is active
// (every lane before fe, the first mask[q] lanes after it).
constexpr int kLavU = 4;  // steps whose loads are in flight together (8 measured slower)

template <class V, class X, class CT, int L>
__device__ __forceinline__ CT lav_steps(int q, int qend, int qstride, int fe, int i, int64_t base, int64_t nmax,
                                        const uint16_t* __restrict__ mk, const V* __restrict__ val,
                                        const uint32_t* __restrict__ col, const X* __restrict__ x, uint64_t pf,
                                        uint64_t pl) {
  CT part = 0;
  for (; q < qend; q += kLavU * qstride) {
    int64_t e[kLavU];
    uint32_t ci[kLavU];
    V vv[kLavU];
    X xv[kLavU];
#pragma unroll
    for (int u = 0; u < kLavU; ++u) e[u] = base + min(q + u * qstride, qend - 1);
#pragma unroll
    for (int u = 0; u < kLavU; ++u) ci[u] = ld_stream(col + e[u] * L + i, pf);
#pragma unroll
    for (int u = 0; u < kLavU; ++u) vv[u] = ld_stream(val + e[u] * L + i, pf);
#pragma unroll
    for (int u = 0; u < kLavU; ++u) xv[u] = ld_keep(x + min((int64_t)ci[u], nmax), pl);
#pragma unroll
    for (int u = 0; u < kLavU; ++u) {
      const int qq = q + u * qstride;
      if (qq < qend && (qq < fe || i < (int)mk[e[u]])) part += (CT)vmul(vv[u], xv[u]);
    }
  }
  return part;
}

template <class V, class X, class CT, int L>
__global__ void __launch_bounds__(256)
lav_fused_kernel(int64_t nseg, int64_t cc, int64_t m, int64_t n, int64_t nlong, const int* __restrict__ co,
                 const int* __restrict__ cf, const uint64_t* __restrict__ sp, const uint16_t* __restrict__ mk,
                 const V* __restrict__ val, const uint32_t* __restrict__ col, const uint8_t* __restrict__ los,
                 const uint32_t* __restrict__ row_order, const X* __restrict__ x, X* __restrict__ y, X alpha) {
  static_assert(32 % L == 0, "a chunk must not straddle warps");
  constexpr int G = 256 / L;
  const uint64_t pf = policy_evict_first(), pl = policy_evict_last();
  const int64_t nmax = n > 0 ? n - 1 : 0;
  if ((int64_t)blockIdx.x < nlong) {
    __shared__ CT red[256];
    const int64_t c = blockIdx.x;
    const int g = threadIdx.x / L, i = threadIdx.x % L;
    CT acc = 0;
    for (int64_t s = 0; s < nseg; ++s) {
      const int64_t sh = (cc + 1) * s;
      const int st = co[sh + c], en = co[sh + c + 1];
      if (st >= en) continue;  // the same for the whole block
      const int fe = cf[s * cc + c];
      red[threadIdx.x] = lav_steps<V, X, CT, L>(st + g, en, G, fe, i, (int64_t)sp[s], nmax, mk, val, col, x, pf, pl);
      __syncthreads();
      if (threadIdx.x < L) {
        const int src = los[(s * cc + c) * L + threadIdx.x];
        CT segsum = 0;
        for (int gg = 0; gg < G; ++gg) segsum += red[gg * L + src];
        acc += segsum;
      }
      __syncthreads();
    }
    const int64_t gs = c * L + threadIdx.x;
    if (threadIdx.x < L && gs < m) {
      const uint32_t r = row_order[gs];
      y[r] += alpha * (X)acc;
    }
    return;
  }
  const int64_t gid = nlong * L + ((int64_t)blockIdx.x - nlong) * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const int64_t c = gid / L;
  const int i = (int)(gid % L);
  const bool live = c < cc;
  CT acc = 0;
  for (int64_t s = 0; s < nseg; ++s) {
    CT part = 0;
    int src = i;
    if (live) {
      const int64_t sh = (cc + 1) * s;
      const int st = co[sh + c], en = co[sh + c + 1];
      if (st < en) {
        src = los[(s * cc + c) * L + i];
        part = lav_steps<V, X, CT, L>(st, en, 1, cf[s * cc + c], i, (int64_t)sp[s], nmax, mk, val, col, x, pf, pl);
      }
    }
    acc += __shfl_sync(0xffffffffu, part, (lane & ~(L - 1)) + src);
  }
  const int64_t g = c * L + i;
  if (live && g < m) {
    const uint32_t r = row_order[g];
    y[r] += alpha * (X)acc;
  }
}

constexpr int64_t kLavLongSteps = 128;


}  // namespace

// lav_build.cu
template <class T>
int lav_build_gpu(const rvvla_crs* src, int64_t L, double Tthr, int64_t seglen, int64_t long_steps,
                  rvvla_lav_owned* out, cudaStream_t st);

namespace {

template <class T>
int lav_build_typed(const rvvla_crs* src, int64_t L, double Tthr, int64_t seglen, rvvla_lav_owned* out, cudaStream_t st) {
  if (src->m > 0 && (!src->Rst || (src->nz > 0 && (!src->Col || !src->Val))))
    return fail(RVVLA_ERR_INVALID_ARG, "lav_build: null array");
  int rc = lav_build_gpu<T>(src, L, Tthr, seglen, kLavLongSteps, out, st);
  if (rc) return rc;
  rvvla_lav& h = out->h;
  const int64_t m = src->m;
  if (h.sparse_part.nz > 0) {  // analyse the sparse part once for the CRS lane-run kernel
    const int dt = sizeof(T) == 8 ? RVVLA_F64 : RVVLA_F32;
    const int64_t plen = rvvla_crs_plan_len(m, h.sparse_part.nz, dt);
    RVVLA_CUDA(cudaMalloc(&out->sp_plan, (size_t)std::max<int64_t>(plen, 1) * sizeof(int32_t)));
    int64_t tiles = 0;
    int32_t kind = 0;
    if ((rc = rvvla_crs_analyze(&h.sparse_part, dt, out->sp_plan, &tiles, &kind, st))) return rc;
    h.sparse_part.plan = out->sp_plan; h.sparse_part.plan_tiles = tiles; h.sparse_part.plan_kind = kind;
  }
  RVVLA_CUDA(cudaStreamSynchronize(st));
  return RVVLA_OK;
}

template <class V, class X, class CT>
int lav_spmv_impl(const rvvla_lav* A, X alpha, const X* x, X beta, X* y, cudaStream_t st,
                  int (*crs_fn)(const rvvla_crs*, X, const X*, X, X*, void*)) {
  if (!A) return fail(RVVLA_ERR_INVALID_ARG, "lav: null descriptor");
  if (A->m < 0 || A->SIMD_Lanes <= 0 || A->segment_count < 0 || A->chunk_count != (A->m + A->SIMD_Lanes - 1) / A->SIMD_Lanes)
    return fail(RVVLA_ERR_INVALID_ARG, "lav: bad sizes");
  if (A->m == 0) return RVVLA_OK;
  // sparse part: y = alpha*S*x + beta*y over every row (spmv_mtx_lav.cpp:31)
  int rc = crs_fn(&A->sparse_part, alpha, x, beta, y, (void*)st);
  if (rc) return rc;
  const int64_t threads = A->chunk_count * A->SIMD_Lanes;
  if (A->segment_count == 0) return RVVLA_OK;
  if (A->row_order && A->lane_of_slot && A->SIMD_Lanes <= 32 && 32 % A->SIMD_Lanes == 0) {
    // long chunks: a multiple of the chunks per warp, so that the rest
    // starts on a warp boundary
    const int64_t cpw = 32 / A->SIMD_Lanes;
    const int64_t nlong = std::min(A->chunk_count, std::max<int64_t>(A->long_chunks, 0) + cpw - 1) / cpw * cpw;
    const int64_t rest = (A->chunk_count - nlong) * A->SIMD_Lanes;
    const int64_t total = (rest + 31) / 32 * 32;  // whole warps: every lane takes part in the shuffles
    const unsigned blocks = (unsigned)(nlong + (total + 255) / 256);
    switch (A->SIMD_Lanes) {
#define LAV_FUSED(LN)                                                                                          \
  case LN:                                                                                                     \
    lav_fused_kernel<V, X, CT, LN><<<blocks, 256, 0, st>>>(A->segment_count, A->chunk_count, A->m, A->n,       \
                                                          nlong,                                              \
                                                          A->chunk_offsets, A->chunk_offsets_full_mask,       \
                                                          A->segment_ptr, A->mask, (const V*)A->val,          \
                                                          A->col_id, A->lane_of_slot, A->row_order, x, y,     \
                                                          alpha);                                             \
    break;
      LAV_FUSED(1)
      LAV_FUSED(2)
      LAV_FUSED(4)
      LAV_FUSED(8)
      LAV_FUSED(16)
      LAV_FUSED(32)
#undef LAV_FUSED
    }
    RVVLA_LAUNCHED("lav_fused_kernel");
    return RVVLA_OK;
  }
  for (int64_t s = 0; s < A->segment_count; ++s) {
    lav_segment_kernel<V, X, CT><<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(
        s, A->SIMD_Lanes, A->chunk_count, A->chunk_offsets, A->chunk_offsets_full_mask, A->segment_ptr, A->out_order,
        A->mask, (const V*)A->val, A->col_id, x, y, alpha);
    RVVLA_LAUNCHED("lav_segment_kernel");
  }
  return RVVLA_OK;
}

}  // namespace
}  // namespace rvvla

using namespace rvvla;

extern "C" {

int rvvla_lav_build(const rvvla_crs* src, int val_bytes, int64_t simd_lanes, double T, int64_t segment_len,
                    rvvla_lav_owned* out, void* stream) {
  if (!src || !out) return fail(RVVLA_ERR_INVALID_ARG, "lav_build: null argument");
  std::memset(out, 0, sizeof(*out));
  if (simd_lanes <= 0 || segment_len <= 0 || simd_lanes > 65535)
    return fail(RVVLA_ERR_INVALID_ARG, "LAV: SIMD_Lanes and segment_len must be positive");
  if (src->m < 0 || src->n < 0 || src->nz < 0) return fail(RVVLA_ERR_INVALID_ARG, "lav_build: bad sizes");
  int rc;
  if (val_bytes == 8) rc = lav_build_typed<double>(src, simd_lanes, T, segment_len, out, as_stream(stream));
  else if (val_bytes == 4) rc = lav_build_typed<float>(src, simd_lanes, T, segment_len, out, as_stream(stream));
  else rc = fail(RVVLA_ERR_INVALID_ARG, "lav_build: val_bytes must be 8 or 4");
  if (rc) {
    std::string keep = rvvla_last_error();
    rvvla_lav_free(out);
    set_error(keep);
  }
  return rc;
}

void rvvla_lav_free(rvvla_lav_owned* h) {
  if (!h) return;
  void* ptrs[] = {h->chunk_offsets, h->chunk_offsets_full_mask, h->segment_ptr, h->out_order, h->mask, h->val,
                  h->col_id, h->sp_Rst, h->sp_Col, h->sp_Val, h->row_order, h->lane_of_slot, h->sp_plan};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  std::memset(h, 0, sizeof(*h));
}

int rvvla_lav_spmv_f64(const rvvla_lav* A, double alpha, const double* x, double beta, double* y, void* stream) {
  return lav_spmv_impl<double, double, double>(A, alpha, x, beta, y, as_stream(stream), rvvla_crs_spmv_f64);
}

int rvvla_lav_spmv_f32(const rvvla_lav* A, float alpha, const float* x, float beta, float* y, void* stream) {
  return lav_spmv_impl<float, float, float>(A, alpha, x, beta, y, as_stream(stream), rvvla_crs_spmv_f32);
}

}  // extern "C"
