// batched.cu — many independent SpMVs (Y_i = alpha * A_i X_i + beta * Y_i,
// each X_i / Y_i holding k right-hand sides) in ONE persistent launch, with a
// CUDA-graph wrapper and a measuring autotuner.  No reference counterpart.
//
// Plan (rvvla_batched_plan): each matrix runs either as CSR (the caller's
// arrays) or as SELL-C-sigma (C = 32, built on the GPU and owned by the
// plan); its rows (CSR) or slices (SELL) are cut into tiles of bounded work,
// and all tiles of all matrices form one list.  The kernel keeps
// sm_count x (resident CTAs per SM) CTAs alive and walks the list with a
// grid stride, so a batch of uneven matrices costs one launch.
//
// Vectors: X_i is n_i x k and Y_i is m_i x k, row-major (the k values of one
// row contiguous), packed one matrix after another; x_off/y_off give each
// matrix's first element.  A nonzero (j, c) of row r then needs the k
// contiguous values X[c*k .. c*k+k-1], one coalesced access per group.
//
// Mappings (per tile, one CTA of 256 threads):
//   CSR, k = 1   tpr lanes per row (tpr in {1,2,4,...,32}, per matrix): lanes
//                stride over the row, shuffle reduction inside the group;
//   CSR, k > 1   k lanes per row (k in {4, 8, 32}), lane = right-hand side;
//                the tile's columns and values (at most 2048 nonzeros) are
//                staged in shared memory with one coalesced pass, then the
//                group walks the row from there, each lane gathering its own
//                X value, 8 nonzeros in flight;
//   SELL, k = 1  a warp per slice, lane = row, column-major loads;
//   SELL, k > 1  a warp per slice, lane = row, k accumulators per lane.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "rvvla_internal.cuh"

namespace rvvla {
namespace {

constexpr int kBThreads = 256;
constexpr int kBWarps = kBThreads / 32;

struct BatchMat {
  const int* Rst;
  const int* Col;
  const void* Val;
  // SELL-C-sigma arrays (mode 1)
  const int* sCl;
  const int* sCs;
  const int* sBs;
  const int* sSBs;
  const uint32_t* sCol;
  const uint32_t* sPerm;
  const void* sVal;
  int64_t x_off, y_off;
  int32_t m, n, mode, tpr;
};

struct BatchTile {
  int32_t mat, first, count, pad;
};

template <class T>
__device__ __forceinline__ void store_y(T* y, T alpha, T beta, T v) {
  *y = (beta == T(0)) ? alpha * v : alpha * v + beta * *y;
}

// The row pointers of the tile are staged in shared memory first (one
// coalesced load), so no row waits on a dependent row-pointer load.
constexpr int kTileRowsMax = 2048;

template <class T>
__device__ void csr_k1(const BatchMat& A, const BatchTile& t, const int* __restrict__ srst, const T* __restrict__ X,
                       T* __restrict__ Y, T alpha, T beta) {
  const int tpr = A.tpr;
  const int slot = threadIdx.x / tpr, lane = threadIdx.x % tpr, nslots = kBThreads / tpr;
  const T* __restrict__ x = X + A.x_off;
  const T* __restrict__ val = static_cast<const T*>(A.Val);
  const uint64_t pf = policy_evict_first(), pl = policy_evict_last();
  // every group of tpr lanes runs the same number of iterations (row count
  // rounded up), so the sub-warp shuffles below are always convergent
  const int iters = (t.count + nslots - 1) / nslots;
  for (int it = 0; it < iters; ++it) {
    const int rr = it * nslots + slot;
    const bool valid = rr < t.count;
    T s0 = T(0), s1 = T(0);
    if (valid) {
      const int b = srst[rr], e = srst[rr + 1];
      int j = b + lane;
      for (; j + tpr < e; j += 2 * tpr) {
        const int c0 = ld_stream(A.Col + j, pf), c1 = ld_stream(A.Col + j + tpr, pf);
        const T v0 = ld_stream(val + j, pf), v1 = ld_stream(val + j + tpr, pf);
        s0 += v0 * ld_keep(x + c0, pl);
        s1 += v1 * ld_keep(x + c1, pl);
      }
      if (j < e) s0 += ld_stream(val + j, pf) * ld_keep(x + ld_stream(A.Col + j, pf), pl);
    }
    T s = s0 + s1;
    for (int off = tpr >> 1; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off, tpr);
    if (valid && lane == 0) store_y(Y + A.y_off + t.first + rr, alpha, beta, s);
  }
}

constexpr int kStageNnz = 2048;  // nonzeros of a k > 1 CSR tile staged in shared memory

template <class T, int K>
__device__ void csr_kn(const BatchMat& A, const BatchTile& t, const int* __restrict__ srst, int* __restrict__ s_col,
                       T* __restrict__ s_val, const T* __restrict__ X, T* __restrict__ Y, T alpha, T beta) {
  constexpr int nslots = kBThreads / K;
  constexpr int U = 8;
  const int slot = threadIdx.x / K, rhs = threadIdx.x % K;
  const T* __restrict__ x = X + A.x_off + rhs;
  const T* __restrict__ val = static_cast<const T*>(A.Val);
  const uint64_t pf = policy_evict_first(), pl = policy_evict_last();
  const int b0 = srst[0], nzt = srst[t.count] - b0;
  // uniform over the CTA (the tile is shared): stage, or read in place (a
  // single row longer than the stage)
  const bool staged = nzt <= kStageNnz;
  if (staged) {
    for (int i = threadIdx.x; i < nzt; i += kBThreads) {
      s_col[i] = ld_stream(A.Col + b0 + i, pf);
      s_val[i] = ld_stream(val + b0 + i, pf);
    }
    __syncthreads();
  }
  for (int rr = slot; rr < t.count; rr += nslots) {
    const int b = srst[rr] - b0, e = srst[rr + 1] - b0;
    T s[U];
#pragma unroll
    for (int u = 0; u < U; ++u) s[u] = T(0);
    int j = b;
    for (; j + U <= e; j += U) {
      int c[U];
      T v[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        c[u] = staged ? s_col[j + u] : A.Col[b0 + j + u];
        v[u] = staged ? s_val[j + u] : val[b0 + j + u];
      }
#pragma unroll
      for (int u = 0; u < U; ++u) s[u] += v[u] * ld_keep(x + (int64_t)c[u] * K, pl);
    }
    for (; j < e; ++j) {
      const int c = staged ? s_col[j] : A.Col[b0 + j];
      const T v = staged ? s_val[j] : val[b0 + j];
      s[0] += v * ld_keep(x + (int64_t)c * K, pl);
    }
    const T r = ((s[0] + s[1]) + (s[2] + s[3])) + ((s[4] + s[5]) + (s[6] + s[7]));
    store_y(Y + A.y_off + (int64_t)(t.first + rr) * K + rhs, alpha, beta, r);
  }
}

// Slice metadata of a SELL tile (height, width, start, first sorted row),
// staged in shared memory so a slice starts without dependent loads.
constexpr int kTileSlicesMax = kBWarps * 4;

template <class T, int K>
__device__ void sell_kn(const BatchMat& A, const BatchTile& t, const int (*meta)[kTileSlicesMax],
                        const T* __restrict__ X, T* __restrict__ Y, T alpha, T beta) {
  constexpr int U = (K == 1) ? 8 : 4;  // columns in flight
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const T* __restrict__ val = static_cast<const T*>(A.sVal);
  const T* __restrict__ x = X + A.x_off;
  const uint64_t pf = policy_evict_first(), pl = policy_evict_last();
  for (int q = warp; q < t.count; q += kBWarps) {
    const int h = meta[0][q], w = meta[1][q], base = meta[2][q];
    if (lane >= h) continue;
    const int row = (int)A.sPerm[meta[3][q] + lane];
    T acc[K];
#pragma unroll
    for (int i = 0; i < K; ++i) acc[i] = T(0);
    int j = 0;
    for (; j + U <= w; j += U) {
      T v[U];
      uint32_t c[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int64_t idx = (int64_t)base + (int64_t)(j + u) * h + lane;
        v[u] = ld_stream(val + idx, pf);
        c[u] = ld_stream(A.sCol + idx, pf);
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const T* xr = x + (int64_t)c[u] * K;
#pragma unroll
        for (int i = 0; i < K; ++i) acc[i] += v[u] * ld_keep(xr + i, pl);
      }
    }
    for (; j < w; ++j) {
      const int64_t idx = (int64_t)base + (int64_t)j * h + lane;
      const T v = ld_stream(val + idx, pf);
      const T* xr = x + (int64_t)ld_stream(A.sCol + idx, pf) * K;
#pragma unroll
      for (int i = 0; i < K; ++i) acc[i] += v * ld_keep(xr + i, pl);
    }
    T* yr = Y + A.y_off + (int64_t)row * K;
#pragma unroll
    for (int i = 0; i < K; ++i) store_y(yr + i, alpha, beta, acc[i]);
  }
}

template <class T, int K>
__global__ void __launch_bounds__(kBThreads)
batched_kernel(int64_t ntiles, const BatchTile* __restrict__ tiles, const BatchMat* __restrict__ mats,
               const T* __restrict__ X, T* __restrict__ Y, T alpha, T beta) {
  // per tile: the matrix entry and the tile's row pointers (CSR) or slice
  // metadata (SELL) are copied to shared memory once, then used by all warps
  __shared__ int srst[kTileRowsMax + 1];
  __shared__ int meta[4][kTileSlicesMax];
  __shared__ int s_col[K > 1 ? kStageNnz : 1];
  __shared__ T s_val[K > 1 ? kStageNnz : 1];
  __shared__ __align__(16) unsigned char sAraw[sizeof(BatchMat)];
  const BatchMat& A = *reinterpret_cast<const BatchMat*>(sAraw);
  static_assert(sizeof(BatchMat) % 8 == 0, "BatchMat is copied as 8-byte words");
  for (int64_t ti = blockIdx.x; ti < ntiles; ti += gridDim.x) {
    const BatchTile t = tiles[ti];
    __syncthreads();  // the previous tile is done with the shared copies
    if (threadIdx.x < (int)(sizeof(BatchMat) / 8))
      reinterpret_cast<uint64_t*>(sAraw)[threadIdx.x] =
          reinterpret_cast<const uint64_t*>(mats + t.mat)[threadIdx.x];
    __syncthreads();
    if (A.mode == 0) {  // uniform over the CTA: the tile is shared
      for (int i = threadIdx.x; i <= t.count; i += kBThreads) srst[i] = A.Rst[t.first + i];
      __syncthreads();
      if constexpr (K == 1) csr_k1<T>(A, t, srst, X, Y, alpha, beta);
      else csr_kn<T, K>(A, t, srst, s_col, s_val, X, Y, alpha, beta);
    } else {
      if (threadIdx.x < t.count) {
        const int sl = t.first + threadIdx.x;
        meta[0][threadIdx.x] = A.sBs[sl];
        meta[1][threadIdx.x] = A.sCl[sl];
        meta[2][threadIdx.x] = A.sCs[sl];
        meta[3][threadIdx.x] = A.sSBs[sl];
      }
      __syncthreads();
      sell_kn<T, K>(A, t, meta, X, Y, alpha, beta);
    }
  }
}

constexpr int64_t kTileWork = 8192;  // k = 1 CSR tile: nonzeros + rows; SELL tile: 4x this in products

int default_tpr(double avg) {
  int t = 1;
  while (t < 32 && t < avg) t <<= 1;
  return std::max(1, t / 2);
}

template <class T>
int batched_launch(const rvvla_batch* B, T alpha, const T* X, T beta, T* Y, cudaStream_t st) {
  if (!B) return fail(RVVLA_ERR_INVALID_ARG, "batched_spmv: null plan");
  if (B->val_bytes != (int)sizeof(T)) return fail(RVVLA_ERR_INVALID_ARG, "batched_spmv: value type differs from the plan");
  if (B->ntiles == 0) return RVVLA_OK;
  if ((B->x_len > 0 && !X) || (B->y_len > 0 && !Y)) return fail(RVVLA_ERR_INVALID_ARG, "batched_spmv: null vectors");
  const auto* tiles = static_cast<const BatchTile*>(B->tiles);
  const auto* mats = static_cast<const BatchMat*>(B->mats);
  switch (B->k) {
    case 1: batched_kernel<T, 1><<<B->grid, kBThreads, 0, st>>>(B->ntiles, tiles, mats, X, Y, alpha, beta); break;
    case 4: batched_kernel<T, 4><<<B->grid, kBThreads, 0, st>>>(B->ntiles, tiles, mats, X, Y, alpha, beta); break;
    case 8: batched_kernel<T, 8><<<B->grid, kBThreads, 0, st>>>(B->ntiles, tiles, mats, X, Y, alpha, beta); break;
    case 32: batched_kernel<T, 32><<<B->grid, kBThreads, 0, st>>>(B->ntiles, tiles, mats, X, Y, alpha, beta); break;
    default: return fail(RVVLA_ERR_INVALID_ARG, "batched_spmv: bad k in plan");
  }
  RVVLA_LAUNCHED("batched_kernel");
  return RVVLA_OK;
}

template <class T>
int resident_ctas(int k) {
  int per_sm = 1;
  auto kern = k == 1 ? batched_kernel<T, 1> : k == 4 ? batched_kernel<T, 4> : k == 8 ? batched_kernel<T, 8>
                                                                                      : batched_kernel<T, 32>;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBThreads, 0) != cudaSuccess) per_sm = 1;
  return std::max(per_sm, 1);
}

// Times one plan: one warm-up launch, then the best of three (CUDA events on
// `st`, zeroed X from the stream-ordered pool).
int time_plan(const rvvla_batch& B, cudaStream_t st, double* ms) {
  *ms = 0.0;
  if (B.ntiles == 0) return RVVLA_OK;
  const size_t vb = (size_t)B.val_bytes;
  Scratch sx, sy;
  RVVLA_CUDA(sx.alloc(std::max<int64_t>(B.x_len, 1) * vb, st));
  RVVLA_CUDA(sy.alloc(std::max<int64_t>(B.y_len, 1) * vb, st));
  RVVLA_CUDA(cudaMemsetAsync(sx.p, 0, std::max<int64_t>(B.x_len, 1) * vb, st));
  cudaEvent_t e0, e1;
  RVVLA_CUDA(cudaEventCreate(&e0));
  RVVLA_CUDA(cudaEventCreate(&e1));
  double best = 1e30;
  int rc = RVVLA_OK;
  for (int it = 0; it < 4 && rc == RVVLA_OK; ++it) {
    cudaEventRecord(e0, st);
    rc = (vb == 8) ? batched_launch<double>(&B, 1.0, sx.as<double>(), 0.0, sy.as<double>(), st)
                   : batched_launch<float>(&B, 1.f, sx.as<float>(), 0.f, sy.as<float>(), st);
    cudaEventRecord(e1, st);
    if (cudaEventSynchronize(e1) != cudaSuccess) rc = fail(RVVLA_ERR_CUDA, "autotune: launch failed");
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    if (it > 0) best = std::min(best, (double)t);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = best;
  return rc;
}

struct BatchGraph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

}  // namespace
}  // namespace rvvla

using namespace rvvla;

extern "C" {

void rvvla_batched_free(rvvla_batch_owned* b) {
  if (!b) return;
  if (b->sell)
    for (int64_t i = 0; i < b->nmats; ++i) rvvla_sell_free(&b->sell[i]);
  if (b->mats) cudaFree(b->mats);
  if (b->tiles) cudaFree(b->tiles);
  std::free(b->x_off);
  std::free(b->y_off);
  std::free(b->sell);
  std::memset(b, 0, sizeof(*b));
}

int rvvla_batched_plan(const rvvla_crs* mats, int64_t count, int val_bytes, int k, const int32_t* mode,
                       const int32_t* param, rvvla_batch_owned* out, void* stream) {
  if (!out) return fail(RVVLA_ERR_INVALID_ARG, "batched_plan: null output");
  std::memset(out, 0, sizeof(*out));
  if (count < 0 || (count > 0 && !mats)) return fail(RVVLA_ERR_INVALID_ARG, "batched_plan: bad matrix list");
  if (val_bytes != 4 && val_bytes != 8) return fail(RVVLA_ERR_INVALID_ARG, "batched_plan: val_bytes must be 4 or 8");
  if (k != 1 && k != 4 && k != 8 && k != 32) return fail(RVVLA_ERR_INVALID_ARG, "batched_plan: k must be 1, 4, 8 or 32");
  cudaStream_t st = as_stream(stream);
  int rc = RVVLA_OK;
  std::vector<BatchMat> tab((size_t)count);
  std::vector<BatchTile> tiles;
  out->x_off = static_cast<int64_t*>(std::calloc((size_t)count + 1, sizeof(int64_t)));
  out->y_off = static_cast<int64_t*>(std::calloc((size_t)count + 1, sizeof(int64_t)));
  out->sell = static_cast<rvvla_sell_owned*>(std::calloc((size_t)std::max<int64_t>(count, 1), sizeof(rvvla_sell_owned)));
  out->nmats = count;
  if (!out->x_off || !out->y_off || !out->sell) {
    rvvla_batched_free(out);
    return fail(RVVLA_ERR_CUDA, "batched_plan: host allocation failed");
  }
  std::vector<int> Rst;
  for (int64_t i = 0; i < count && rc == RVVLA_OK; ++i) {
    const rvvla_crs& A = mats[i];
    if (A.m < 0 || A.n < 0 || A.nz < 0 || A.m >= INT32_MAX || A.n >= INT32_MAX || A.nz >= INT32_MAX ||
        (A.m > 0 && !A.Rst) || (A.nz > 0 && (!A.Col || !A.Val))) {
      rc = fail(RVVLA_ERR_INVALID_ARG, "batched_plan: matrix " + std::to_string(i) + " has bad sizes or arrays");
      break;
    }
    BatchMat& b = tab[(size_t)i];
    std::memset(&b, 0, sizeof(b));
    b.Rst = A.Rst; b.Col = A.Col; b.Val = A.Val;
    b.m = (int32_t)A.m; b.n = (int32_t)A.n;
    b.x_off = out->x_off[i];
    b.y_off = out->y_off[i];
    out->x_off[i + 1] = out->x_off[i] + A.n * k;
    out->y_off[i + 1] = out->y_off[i] + A.m * k;
    if (A.m == 0) continue;
    Rst.resize((size_t)A.m + 1);
    if (cudaMemcpyAsync(Rst.data(), A.Rst, (A.m + 1) * sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
      rc = fail(RVVLA_ERR_CUDA, "batched_plan: reading row pointers failed");
      break;
    }
    const int md = mode ? mode[i] : 0;
    const double avg = (double)A.nz / (double)A.m;
    if (md == 0) {
      b.mode = 0;
      const int tpr = (param && param[i] > 0) ? param[i] : default_tpr(avg);
      if (tpr > 32 || (tpr & (tpr - 1))) {
        rc = fail(RVVLA_ERR_INVALID_ARG, "batched_plan: threads per row must be a power of two <= 32");
        break;
      }
      b.tpr = (k == 1) ? tpr : k;
      // tiles of whole rows: k = 1 at most kTileWork nonzeros and 8 row
      // passes of the CTA; k > 1 at most the staged nonzeros and 32 passes
      const int64_t max_rows = std::min<int64_t>((int64_t)(kBThreads / b.tpr) * (k == 1 ? 8 : 32), kTileRowsMax);
      const int64_t max_work = k == 1 ? kTileWork : kStageNnz;
      int64_t r0 = 0;
      while (r0 < A.m) {
        int64_t r1 = r0, work = 0;
        while (r1 < A.m && r1 - r0 < max_rows) {
          const int64_t wr = (int64_t)Rst[(size_t)r1 + 1] - Rst[(size_t)r1] + (k == 1 ? 1 : 0);
          if (r1 > r0 && work + wr > max_work) break;
          work += wr;
          ++r1;
        }
        tiles.push_back({(int32_t)i, (int32_t)r0, (int32_t)(r1 - r0), 0});
        r0 = r1;
      }
    } else if (md == 1) {
      b.mode = 1;
      const int sigma = (param && param[i] > 0) ? param[i] : 256;
      rvvla_crs src = A;
      src.plan = nullptr;
      src.plan_tiles = 0;
      src.plan_kind = 0;
      rc = rvvla_sell_build(&src, val_bytes, 32, sigma, &out->sell[i], stream);
      if (rc) break;
      const rvvla_sell& s = out->sell[i].h;
      b.sCl = s.vCl; b.sCs = s.vCs; b.sBs = s.vBs; b.sSBs = s.vSBs;
      b.sCol = s.vCol; b.sPerm = s.vPerm; b.sVal = s.vVal;
      std::vector<int> Cl((size_t)s.cnt_b);
      if (s.cnt_b && (cudaMemcpy(Cl.data(), s.vCl, s.cnt_b * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)) {
        rc = fail(RVVLA_ERR_CUDA, "batched_plan: reading slice widths failed");
        break;
      }
      int64_t q0 = 0;
      while (q0 < s.cnt_b) {
        int64_t q1 = q0, work = 0;
        while (q1 < s.cnt_b && q1 - q0 < kTileSlicesMax) {
          const int64_t wq = ((int64_t)Cl[(size_t)q1] + 1) * 32 * k;
          if (q1 > q0 && work + wq > 4 * kTileWork) break;
          work += wq;
          ++q1;
        }
        tiles.push_back({(int32_t)i, (int32_t)q0, (int32_t)(q1 - q0), 0});
        q0 = q1;
      }
    } else {
      rc = fail(RVVLA_ERR_INVALID_ARG, "batched_plan: mode must be 0 (CSR) or 1 (SELL)");
      break;
    }
  }
  if (rc) {
    std::string keep = rvvla_last_error();
    rvvla_batched_free(out);
    set_error(keep);
    return rc;
  }
  rvvla_batch& h = out->h;
  h.count = count;
  h.k = k;
  h.val_bytes = val_bytes;
  h.x_len = out->x_off[count];
  h.y_len = out->y_off[count];
  h.ntiles = (int64_t)tiles.size();
  auto fail_cuda = [&](cudaError_t e, const char* where) {
    const int r = cuda_fail(e, where);
    std::string keep = rvvla_last_error();
    rvvla_batched_free(out);
    set_error(keep);
    return r;
  };
  cudaError_t e;
  if ((e = cudaMalloc(&out->mats, std::max<size_t>(tab.size(), 1) * sizeof(BatchMat))) != cudaSuccess)
    return fail_cuda(e, "cudaMalloc(mats)");
  if ((e = cudaMalloc(&out->tiles, std::max<size_t>(tiles.size(), 1) * sizeof(BatchTile))) != cudaSuccess)
    return fail_cuda(e, "cudaMalloc(tiles)");
  if (!tab.empty() &&
      (e = cudaMemcpyAsync(out->mats, tab.data(), tab.size() * sizeof(BatchMat), cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return fail_cuda(e, "cudaMemcpyAsync(mats)");
  if (!tiles.empty() && (e = cudaMemcpyAsync(out->tiles, tiles.data(), tiles.size() * sizeof(BatchTile),
                                             cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return fail_cuda(e, "cudaMemcpyAsync(tiles)");
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail_cuda(e, "cudaStreamSynchronize");
  // persistent grid: every SM filled with as many CTAs as fit
  const int per_sm = (val_bytes == 8) ? resident_ctas<double>(k) : resident_ctas<float>(k);
  h.grid = (int32_t)std::max<int64_t>(1, std::min<int64_t>((int64_t)sm_count() * per_sm, h.ntiles));
  h.block = kBThreads;
  h.mats = out->mats;
  h.tiles = out->tiles;
  return RVVLA_OK;
}

int rvvla_batched_spmv_f64(const rvvla_batch* B, double alpha, const double* X, double beta, double* Y, void* stream) {
  return batched_launch<double>(B, alpha, X, beta, Y, as_stream(stream));
}

int rvvla_batched_spmv_f32(const rvvla_batch* B, float alpha, const float* X, float beta, float* Y, void* stream) {
  return batched_launch<float>(B, alpha, X, beta, Y, as_stream(stream));
}

int rvvla_batched_graph(const rvvla_batch* B, double alpha, const void* X, double beta, void* Y, void* stream,
                        void** graph) {
  if (!B || !graph) return fail(RVVLA_ERR_INVALID_ARG, "batched_graph: null argument");
  *graph = nullptr;
  cudaStream_t st = as_stream(stream);
  if (!st) return fail(RVVLA_ERR_INVALID_ARG, "batched_graph: capture needs a non-default stream");
  auto* g = new BatchGraph();
  const cudaError_t eb = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
  if (eb != cudaSuccess) {
    delete g;
    return cuda_fail(eb, "cudaStreamBeginCapture");
  }
  const int rc = (B->val_bytes == 8)
                     ? batched_launch<double>(B, alpha, static_cast<const double*>(X), beta, static_cast<double*>(Y), st)
                     : batched_launch<float>(B, (float)alpha, static_cast<const float*>(X), (float)beta,
                                             static_cast<float*>(Y), st);
  const cudaError_t ec = cudaStreamEndCapture(st, &g->graph);
  if (rc || ec != cudaSuccess) {
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
    return rc ? rc : cuda_fail(ec, "cudaStreamEndCapture");
  }
  const cudaError_t ei = cudaGraphInstantiate(&g->exec, g->graph, 0);
  if (ei != cudaSuccess) {
    cudaGraphDestroy(g->graph);
    delete g;
    return cuda_fail(ei, "cudaGraphInstantiate");
  }
  *graph = g;
  return RVVLA_OK;
}

int rvvla_batched_graph_launch(void* graph, void* stream) {
  if (!graph) return fail(RVVLA_ERR_INVALID_ARG, "batched_graph_launch: null graph");
  auto* g = static_cast<BatchGraph*>(graph);
  RVVLA_CUDA(cudaGraphLaunch(g->exec, as_stream(stream)));
  count_launch(1);
  return RVVLA_OK;
}

void rvvla_batched_graph_free(void* graph) {
  if (!graph) return;
  auto* g = static_cast<BatchGraph*>(graph);
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  delete g;
}

int rvvla_batched_autotune(const rvvla_crs* mats, int64_t count, int val_bytes, int k, int32_t* mode, int32_t* param,
                           double* tuned_ms, void* stream) {
  if (count < 0 || (count > 0 && (!mats || !mode || !param)))
    return fail(RVVLA_ERR_INVALID_ARG, "batched_autotune: null argument");
  if (tuned_ms) *tuned_ms = 0.0;
  cudaStream_t st = as_stream(stream);
  // groups by average row length: [0,2), [2,4), [4,8), ... [128, inf)
  constexpr int kGroups = 8;
  std::vector<std::vector<int64_t>> groups(kGroups);
  for (int64_t i = 0; i < count; ++i) {
    const double avg = mats[i].m > 0 ? (double)mats[i].nz / (double)mats[i].m : 0.0;
    int g = 0;
    while (g + 1 < kGroups && avg >= (double)(2 << g)) ++g;
    groups[(size_t)g].push_back(i);
  }
  struct Cand {
    int32_t mode, param;
  };
  std::vector<Cand> cands;
  if (k == 1)
    for (int t = 1; t <= 32; t <<= 1) cands.push_back({0, t});
  else
    cands.push_back({0, 0});
  cands.push_back({1, 32});
  cands.push_back({1, 256});
  double total = 0.0;
  for (const auto& grp : groups) {
    if (grp.empty()) continue;
    std::vector<rvvla_crs> sub;
    for (int64_t i : grp) sub.push_back(mats[i]);
    double best = 1e30;
    Cand pick = cands[0];
    for (const Cand& c : cands) {
      std::vector<int32_t> md(sub.size(), c.mode), pr(sub.size(), c.param);
      rvvla_batch_owned plan;
      int rc = rvvla_batched_plan(sub.data(), (int64_t)sub.size(), val_bytes, k, md.data(), pr.data(), &plan, stream);
      if (rc) return rc;
      double ms = 0.0;
      rc = time_plan(plan.h, st, &ms);
      rvvla_batched_free(&plan);
      if (rc) return rc;
      if (ms < best) {
        best = ms;
        pick = c;
      }
    }
    for (int64_t i : grp) {
      mode[i] = pick.mode;
      param[i] = pick.param;
    }
    total += best;
  }
  if (tuned_ms) *tuned_ms = total;
  return RVVLA_OK;
}

}  // extern "C"
