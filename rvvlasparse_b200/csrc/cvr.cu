// cvr.cu — spMtxCVR on sm_100a: GPU builder (SIMD_LEN 32) and SpMV.
//
// Layout (include/CVR.h:22-37 of the reference) as read by
// src/scalar/spmv_mtx_cvr.cpp:32-66: SIMD_LEN lanes stream the nonzeros of
// one row after another (vPack_vec_vals/cols); vPack_vec_record holds
// (pos, row) pairs sorted by pos — before accumulating the vector that holds
// pos, lane pos % SIMD_LEN is flushed into y[row] — plus one trailing pair;
// writeback_pos_record holds Nthreads blocks of SIMD_LEN+2 ints
// {first vector, first record pair, tail row of each lane}, the last block's
// tail rows are flushed after the final vector.  The reference ships no
// builder; this one reproduces the oracle's: threads own whole-row ranges
// balanced by nonzeros, rows enter lanes longest first (stable), empty rows
// are skipped, lanes still holding a row at a range end get a record at the
// next range's first vector.
//
// SpMV: y *= beta first (as the reference, :115-117), then one warp per
// range (lane = CVR lane): coalesced 32-wide vector loads (L2 evict-first),
// x gathers (evict-last), and per batch of vectors the records that fall in
// it are scattered to their (vector, lane) slots through a shared table; a
// flush is y[row] += alpha * lane_sum.  Each row is flushed by one lane once
// (zero sums, e.g. idle tail lanes, are skipped), so the flush is an atomic
// add with a single contributor: deterministic.
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cstring>
#include <string>

#include "crs_merge.cuh"
#include "rvvla_internal.cuh"
#include "scan.cuh"

namespace rvvla {
namespace {

constexpr int kS = 32;  // SIMD_LEN

// ---------------------------------------------------------------- builder
__global__ void cvr_bounds_kernel(int64_t NT, int64_t m, int64_t nnz, const int* __restrict__ Rst,
                                  int64_t* __restrict__ bounds) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t > NT) return;
  if (t == 0) { bounds[0] = 0; return; }
  if (t == NT) { bounds[NT] = m; return; }
  const int64_t target = nnz * t / NT;  // largest r with Rst[r] <= target
  int64_t lo = 0, hi = m + 1;
  while (hi - lo > 1) {
    const int64_t mid = (lo + hi) >> 1;
    if (Rst[mid] <= target) lo = mid;
    else hi = mid;
  }
  bounds[t] = lo;
}

__global__ void cvr_monotone_kernel(int64_t NT, int64_t* __restrict__ bounds) {
  for (int64_t t = 1; t <= NT; ++t) bounds[t] = max(bounds[t], bounds[t - 1]);
}

// sort key: part-major, length descending; rows of a part are contiguous, so
// the part of row r is found by the part bounds.
__global__ void cvr_keys_kernel(int64_t m, int64_t NT, const int* __restrict__ Rst, const int64_t* __restrict__ bounds,
                                uint64_t* __restrict__ key, uint32_t* __restrict__ idx) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= m) return;
  int64_t lo = 0, hi = NT;  // part p with bounds[p] <= r < bounds[p+1]
  while (hi - lo > 1) {
    const int64_t mid = (lo + hi) >> 1;
    if (bounds[mid] <= r) lo = mid;
    else hi = mid;
  }
  const uint32_t len = (uint32_t)(Rst[r + 1] - Rst[r]);
  key[r] = ((uint64_t)lo << 32) | (uint64_t)(0xFFFFFFFFu - len);
  idx[r] = (uint32_t)r;
}

// Replays the lane schedule of one range.  WRITE = false: counts vectors and
// record pairs; WRITE = true: writes them at the scanned offsets.
template <bool WRITE, int VB>
__global__ void cvr_sim_kernel(int64_t NT, const int* __restrict__ Rst, const int* __restrict__ Col,
                               const uint8_t* __restrict__ Val, const int64_t* __restrict__ bounds,
                               const uint32_t* __restrict__ order, int64_t* __restrict__ nvec,
                               int64_t* __restrict__ nrec, const int64_t* __restrict__ vofs,
                               const int64_t* __restrict__ rofs, uint8_t* __restrict__ vals,
                               uint32_t* __restrict__ cols, int* __restrict__ rec, int* __restrict__ wb) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= NT) return;
  int lrow[kS];
  int64_t lpos[kS], lend[kS];
  for (int l = 0; l < kS; ++l) { lrow[l] = -1; lpos[l] = lend[l] = 0; }
  const int64_t r0 = bounds[t], r1 = bounds[t + 1];
  int64_t next = r0;
  // rows of the range are sorted longest first, so empty rows come last
  auto rows_left = [&]() -> bool {
    if (next >= r1) return false;
    const int r = (int)order[next];
    return Rst[r + 1] > Rst[r];
  };
  int64_t nv = WRITE ? vofs[t] : 0;
  int64_t nr = WRITE ? rofs[t] : 0;
  if (WRITE) {
    int* blk = wb + t * (kS + 2);
    blk[0] = (int)nv;
    blk[1] = (int)nr;
  }
  for (;;) {
    bool any = false;
    for (int l = 0; l < kS; ++l) {
      if (lrow[l] >= 0 && lpos[l] == lend[l]) {
        if (WRITE) { rec[2 * nr] = (int)(nv * kS + l); rec[2 * nr + 1] = lrow[l]; }
        nr++;
        lrow[l] = -1;
      }
      if (lrow[l] < 0 && rows_left()) {
        const int r = (int)order[next++];
        lrow[l] = r;
        lpos[l] = Rst[r];
        lend[l] = Rst[r + 1];
      }
      any |= lrow[l] >= 0;
    }
    if (!any) break;
    for (int l = 0; l < kS; ++l) {
      const int64_t q = nv * kS + l;
      if (lrow[l] >= 0 && lpos[l] < lend[l]) {
        if (WRITE) {
          cols[q] = (uint32_t)Col[lpos[l]];
          for (int b = 0; b < VB; ++b) vals[q * VB + b] = Val[lpos[l] * VB + b];
        }
        lpos[l]++;
      } else if (WRITE) {
        cols[q] = 0u;
        for (int b = 0; b < VB; ++b) vals[q * VB + b] = 0;
      }
    }
    nv++;
    if (!rows_left()) {
      bool pending = false;
      for (int l = 0; l < kS; ++l) pending |= (lrow[l] >= 0 && lpos[l] < lend[l]);
      if (!pending) break;
    }
  }
  for (int l = 0; l < kS; ++l) {
    const int r = lrow[l];
    if (t + 1 < NT) {
      if (r >= 0) {
        if (WRITE) { rec[2 * nr] = (int)(nv * kS + l); rec[2 * nr + 1] = r; }
        nr++;
      }
      if (WRITE) wb[t * (kS + 2) + 2 + l] = 0;
    } else if (WRITE) {
      wb[t * (kS + 2) + 2 + l] = r >= 0 ? r : 0;
    }
  }
  if (!WRITE) {
    nvec[t] = nv;
    nrec[t] = nr;
  }
}

__global__ void cvr_empty_kernel(int64_t m, const int* __restrict__ Rst, int* __restrict__ flag) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r < m && Rst[r + 1] == Rst[r]) atomicOr(flag, 1);
}

// ---------------------------------------------------------------- SpMV
template <class X>
__global__ void cvr_scale_kernel(int64_t m, X* __restrict__ y, X beta) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) y[i] = (beta == X(0)) ? X(0) : y[i] * beta;
}

// A warp per CVR thread (lane = SIMD lane), cvr_batch<V>() vectors per batch.  A
// batch first issues all loads of its vectors (indices past the range are
// clamped to its last vector and their products dropped), then marks the
// records that fall in the batch in a per-warp table (vector in batch, lane)
// -> row, then each lane walks the batch's vectors: flush into the marked row
// (the record's position is the lane's first slot after the row), add the
// product.  Records come from a 32-entry register window (lane l holds
// record window_base + l) with the next window prefetched.  A row belongs to
// one lane of one range, so each row of y receives exactly one contribution:
// y was scaled by beta first and the flush is a fire-and-forget atomic add
// (no read of y on the critical path, and still deterministic).  Vectors per
// batch: 8 for 8-byte values, 16 for 4-byte ones (about the same bytes in
// flight).
template <class V> constexpr int cvr_batch() { return sizeof(V) >= 8 ? 8 : 16; }

template <class V, class X, class CT>
__global__ void __launch_bounds__(256, 3)
cvr_spmv_kernel(int64_t NT, int64_t nItems, int64_t nrec, const V* __restrict__ vals,
                const uint32_t* __restrict__ cols, const int* __restrict__ rec, const int* __restrict__ wb,
                const X* __restrict__ x, X* __restrict__ y, X alpha) {
  constexpr int kCvrU = cvr_batch<V>();
  __shared__ int s_row[8][kCvrU][kS];
  const int64_t t = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (t >= NT) return;
  const int64_t vb = wb[t * (kS + 2)], rb = wb[t * (kS + 2) + 1];
  const int64_t ve = (t + 1 < NT) ? wb[(t + 1) * (kS + 2)] : nItems / kS;
  const int64_t re = (t + 1 < NT) ? wb[(t + 1) * (kS + 2) + 1] : nrec;
  const uint64_t pf = policy_evict_first(), pl = policy_evict_last();
  CT res = 0;
#pragma unroll
  for (int u = 0; u < kCvrU; ++u) s_row[w][u][lane] = -1;
  // record window and its successor
  auto avail = [&](int64_t base) { return (int)(re - base < 0 ? 0 : (re - base > kS ? kS : re - base)); };
  int64_t wbase = rb;
  int cons = 0;
  int navail = avail(wbase);
  int my_pos = lane < navail ? rec[2 * (wbase + lane)] : INT_MAX;
  int my_row = lane < navail ? rec[2 * (wbase + lane) + 1] : -1;
  int nx_avail = avail(wbase + kS);
  int nx_pos = lane < nx_avail ? rec[2 * (wbase + kS + lane)] : INT_MAX;
  int nx_row = lane < nx_avail ? rec[2 * (wbase + kS + lane) + 1] : -1;
  // mark the records before `limit` whose vector lies in [base, base + kCvrU)
  auto mark = [&](int64_t limit, int64_t base) {
    for (;;) {
      if (cons == navail) {
        if (navail < kS) return;  // no records left in this range
        wbase += kS;
        cons = 0;
        navail = nx_avail;
        my_pos = nx_pos;
        my_row = nx_row;
        if (navail == 0) return;
        nx_avail = avail(wbase + kS);
        nx_pos = lane < nx_avail ? rec[2 * (wbase + kS + lane)] : INT_MAX;
        nx_row = lane < nx_avail ? rec[2 * (wbase + kS + lane) + 1] : -1;
      }
      const bool take = lane >= cons && lane < navail && (int64_t)my_pos < limit;
      const unsigned mk = __ballot_sync(0xffffffffu, take);
      if (take) {
        const int64_t u = (int64_t)my_pos / kS - base;
        if (u >= 0 && u < kCvrU) s_row[w][u][my_pos % kS] = my_row;
      }
      cons += __popc(mk);
      if (cons < navail) return;  // stopped at a record past the limit
    }
  };
  auto flush_batch = [&](int nu, const CT* p) {
    __syncwarp();
#pragma unroll
    for (int u = 0; u < kCvrU; ++u) {
      const int r = s_row[w][u][lane];
      if (r >= 0) {
        if (res != CT(0)) atomicAdd(y + r, alpha * (X)res);
        res = 0;
        s_row[w][u][lane] = -1;
      }
      if (u < nu) res += p[u];
    }
    __syncwarp();
  };
  int64_t v = vb;
  for (; v < ve; v += kCvrU) {
    uint32_t c[kCvrU];
    V a[kCvrU];
    X xv[kCvrU];
#pragma unroll
    for (int u = 0; u < kCvrU; ++u) c[u] = ld_stream(cols + min(v + u, ve - 1) * kS + lane, pf);
#pragma unroll
    for (int u = 0; u < kCvrU; ++u) a[u] = ld_stream(vals + min(v + u, ve - 1) * kS + lane, pf);
#pragma unroll
    for (int u = 0; u < kCvrU; ++u) xv[u] = ld_keep(x + c[u], pl);
    mark((v + kCvrU) * kS, v);
    CT p[kCvrU];
#pragma unroll
    for (int u = 0; u < kCvrU; ++u) p[u] = (CT)vmul(a[u], xv[u]);
    flush_batch(ve - v < kCvrU ? (int)(ve - v) : kCvrU, p);
  }
  // records left: the range-end flushes at vector ve (one batch suffices for
  // well-formed records; later ones take further batches)
  CT none[kCvrU];
#pragma unroll
  for (int u = 0; u < kCvrU; ++u) none[u] = 0;
  for (int guard = 0; guard < 64; ++guard) {
    if (cons == navail && navail < kS) break;
    const int64_t p0 = __shfl_sync(0xffffffffu, my_pos, cons < kS ? cons : 0);
    if (cons == navail) {  // window used up: reload through mark
      mark(v * kS, v);
      continue;
    }
    v = p0 / kS > v ? p0 / kS : v;
    mark((v + kCvrU) * kS, v);
    flush_batch(0, none);
    v += kCvrU;
  }
  if (t + 1 == NT) {  // the last range's tail rows
    const int r = wb[t * (kS + 2) + 2 + lane];
    if (res != CT(0)) atomicAdd(y + r, alpha * (X)res);
  }
}

int cvr_validate(const rvvla_cvr* A, const void* x, const void* y) {
  if (!A) return fail(RVVLA_ERR_INVALID_ARG, "cvr: null descriptor");
  if (A->numRows < 0 || A->Nthreads_avail <= 0 || A->nItems < 0) return fail(RVVLA_ERR_INVALID_ARG, "cvr: bad sizes");
  if (A->SIMD_LEN != kS) return fail(RVVLA_ERR_UNSUPPORTED, "cvr: the sm_100a kernel needs SIMD_LEN 32 (one lane per warp lane)");
  if (A->numRows > 0 && (!A->writeback_pos_record || !y)) return fail(RVVLA_ERR_INVALID_ARG, "cvr: null array");
  if (A->nItems > 0 && (!A->vPack_vec_vals || !A->vPack_vec_cols || !x)) return fail(RVVLA_ERR_INVALID_ARG, "cvr: null array");
  return RVVLA_OK;
}

template <class V, class X, class CT>
int cvr_spmv_impl(const rvvla_cvr* A, X alpha, const X* x, X beta, X* y, cudaStream_t st) {
  int rc = cvr_validate(A, x, y);
  if (rc) return rc;
  if (A->numRows == 0) return RVVLA_OK;
  cvr_scale_kernel<X><<<(unsigned)((A->numRows + 255) / 256), 256, 0, st>>>(A->numRows, y, beta);
  RVVLA_LAUNCHED("cvr_scale_kernel");
  const int64_t NT = A->Nthreads_avail;
  const int64_t nrec = (A->n_record - 2) / 2;
  cvr_spmv_kernel<V, X, CT><<<(unsigned)((NT * 32 + 255) / 256), 256, 0, st>>>(
      NT, A->nItems, nrec, (const V*)A->vPack_vec_vals, A->vPack_vec_cols, A->vPack_vec_record,
      A->writeback_pos_record, x, y, alpha);
  RVVLA_LAUNCHED("cvr_spmv_kernel");
  return RVVLA_OK;
}

int cvr_build_impl(const rvvla_crs* src, int vb, int64_t NT, rvvla_cvr_owned* out, cudaStream_t st) {
  if (!src || !out) return fail(RVVLA_ERR_INVALID_ARG, "cvr_build: null argument");
  std::memset(out, 0, sizeof(*out));
  if (vb != 8 && vb != 4 && vb != 2) return fail(RVVLA_ERR_INVALID_ARG, "cvr_build: val_bytes must be 8, 4 or 2");
  const int64_t m = src->m, nnz = src->nz;
  if (m < 0 || nnz < 0 || src->n < 0) return fail(RVVLA_ERR_INVALID_ARG, "cvr_build: bad sizes");
  // ranges of ~16K nonzeros: smaller ranges drain their lanes unevenly and
  // pad the vectors (4K nonzeros per range double the stored items of a
  // power-law matrix, 8K add ~40 %, 16K ~10 %, 32K ~2 %), larger ones leave
  // too few warps to hide the memory latency (rounding the count to whole
  // waves of resident warps measured no faster)
  if (NT <= 0) NT = std::max<int64_t>(1, (nnz + 16383) / 16384);
  if (nnz >= INT32_MAX / 2 || m >= INT32_MAX) return fail(RVVLA_ERR_TOO_LARGE, "cvr_build: sizes beyond int32 records");
  rvvla_cvr& h = out->h;
  h.numRows = m; h.numCols = src->n; h.SIMD_LEN = kS; h.Nthreads = (int32_t)NT; h.Nthreads_avail = (int32_t)NT;
  Scratch s_b, s_key, s_key2, s_idx, s_ord, s_tmp, s_nv, s_nr, s_vo, s_ro, s_fl;
  RVVLA_CUDA(s_b.alloc((size_t)(NT + 1) * 8, st));
  cvr_bounds_kernel<<<(unsigned)((NT + 1 + 255) / 256), 256, 0, st>>>(NT, m, nnz, src->Rst, s_b.as<int64_t>());
  RVVLA_LAUNCHED("cvr_bounds_kernel");
  cvr_monotone_kernel<<<1, 1, 0, st>>>(NT, s_b.as<int64_t>());
  RVVLA_LAUNCHED("cvr_monotone_kernel");
  RVVLA_CUDA(s_ord.alloc((size_t)std::max<int64_t>(m, 1) * 4, st));
  RVVLA_CUDA(s_fl.alloc(sizeof(int), st));
  RVVLA_CUDA(cudaMemsetAsync(s_fl.p, 0, sizeof(int), st));
  if (m > 0) {
    RVVLA_CUDA(s_key.alloc((size_t)m * 8, st));
    RVVLA_CUDA(s_key2.alloc((size_t)m * 8, st));
    RVVLA_CUDA(s_idx.alloc((size_t)m * 4, st));
    cvr_keys_kernel<<<(unsigned)((m + 255) / 256), 256, 0, st>>>(m, NT, src->Rst, s_b.as<int64_t>(),
                                                                  s_key.as<uint64_t>(), s_idx.as<uint32_t>());
    RVVLA_LAUNCHED("cvr_keys_kernel");
    int end_bit = 33;
    for (int64_t w = NT; w > 1; w >>= 1) end_bit++;
    end_bit = std::min(64, end_bit);
    size_t tb = 0;
    RVVLA_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, s_key.as<uint64_t>(), s_key2.as<uint64_t>(),
                                               s_idx.as<uint32_t>(), s_ord.as<uint32_t>(), (int)m, 0, end_bit, st));
    RVVLA_CUDA(s_tmp.alloc(tb, st));
    RVVLA_CUDA(cub::DeviceRadixSort::SortPairs(s_tmp.p, tb, s_key.as<uint64_t>(), s_key2.as<uint64_t>(),
                                               s_idx.as<uint32_t>(), s_ord.as<uint32_t>(), (int)m, 0, end_bit, st));
    count_launch(3);
    cvr_empty_kernel<<<(unsigned)((m + 255) / 256), 256, 0, st>>>(m, src->Rst, s_fl.as<int>());
    RVVLA_LAUNCHED("cvr_empty_kernel");
  }
  RVVLA_CUDA(s_nv.alloc((size_t)(NT + 1) * 8, st));
  RVVLA_CUDA(s_nr.alloc((size_t)(NT + 1) * 8, st));
  RVVLA_CUDA(s_vo.alloc((size_t)(NT + 1) * 8, st));
  RVVLA_CUDA(s_ro.alloc((size_t)(NT + 1) * 8, st));
  cvr_sim_kernel<false, 8><<<(unsigned)((NT + 63) / 64), 64, 0, st>>>(
      NT, src->Rst, src->Col, nullptr, s_b.as<int64_t>(), s_ord.as<uint32_t>(), s_nv.as<int64_t>(), s_nr.as<int64_t>(),
      nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
  RVVLA_LAUNCHED("cvr_sim_kernel(count)");
  int rc = exclusive_scan_i64(s_nv.as<int64_t>(), s_vo.as<int64_t>(), NT, st);
  if (rc) return rc;
  rc = exclusive_scan_i64(s_nr.as<int64_t>(), s_ro.as<int64_t>(), NT, st);
  if (rc) return rc;
  int64_t tv = 0, tr = 0;
  int any_empty = 0;
  RVVLA_CUDA(cudaMemcpyAsync(&tv, s_vo.as<int64_t>() + NT, 8, cudaMemcpyDeviceToHost, st));
  RVVLA_CUDA(cudaMemcpyAsync(&tr, s_ro.as<int64_t>() + NT, 8, cudaMemcpyDeviceToHost, st));
  RVVLA_CUDA(cudaMemcpyAsync(&any_empty, s_fl.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  RVVLA_CUDA(cudaStreamSynchronize(st));
  if (tv * kS >= INT32_MAX) return fail(RVVLA_ERR_TOO_LARGE, "cvr_build: packed size beyond int32 positions");
  h.nItems = tv * kS;
  h.n_record = 2 * tr + 2;
  h.n_writeback = NT * (kS + 2);
  RVVLA_CUDA(cudaMalloc(&out->vPack_vec_vals, (size_t)std::max<int64_t>(h.nItems, 1) * vb));
  RVVLA_CUDA(cudaMalloc(&out->vPack_vec_cols, (size_t)std::max<int64_t>(h.nItems, 1) * 4));
  RVVLA_CUDA(cudaMalloc(&out->vPack_vec_record, (size_t)h.n_record * 4));
  RVVLA_CUDA(cudaMalloc(&out->writeback_pos_record, (size_t)h.n_writeback * 4));
  const int tail[2] = {(int)h.nItems, 0};
  RVVLA_CUDA(cudaMemcpyAsync(out->vPack_vec_record + 2 * tr, tail, 8, cudaMemcpyHostToDevice, st));
  const unsigned blocks = (unsigned)((NT + 63) / 64);
#define CVR_FILL(VBv)                                                                                              \
  cvr_sim_kernel<true, VBv><<<blocks, 64, 0, st>>>(NT, src->Rst, src->Col, (const uint8_t*)src->Val,                  \
                                                   s_b.as<int64_t>(), s_ord.as<uint32_t>(), nullptr, nullptr,       \
                                                   s_vo.as<int64_t>(), s_ro.as<int64_t>(),                          \
                                                   (uint8_t*)out->vPack_vec_vals, out->vPack_vec_cols,              \
                                                   out->vPack_vec_record, out->writeback_pos_record)
  if (vb == 8) CVR_FILL(8);
  else if (vb == 4) CVR_FILL(4);
  else CVR_FILL(2);
#undef CVR_FILL
  RVVLA_LAUNCHED("cvr_sim_kernel(fill)");
  h.no_empty_rows = any_empty ? 0 : 1;
  h.vPack_vec_vals = out->vPack_vec_vals; h.vPack_vec_cols = out->vPack_vec_cols;
  h.vPack_vec_record = out->vPack_vec_record; h.writeback_pos_record = out->writeback_pos_record;
  RVVLA_CUDA(cudaStreamSynchronize(st));
  return RVVLA_OK;
}

}  // namespace
}  // namespace rvvla

using namespace rvvla;

extern "C" {

int rvvla_cvr_build(const rvvla_crs* src, int val_bytes, int64_t nthreads, rvvla_cvr_owned* out, void* stream) {
  int rc = cvr_build_impl(src, val_bytes, nthreads, out, as_stream(stream));
  if (rc && out) {
    std::string keep = rvvla_last_error();
    rvvla_cvr_free(out);
    set_error(keep);
  }
  return rc;
}

void rvvla_cvr_free(rvvla_cvr_owned* h) {
  if (!h) return;
  cudaFree(h->vPack_vec_vals);
  cudaFree(h->vPack_vec_cols);
  cudaFree(h->vPack_vec_record);
  cudaFree(h->writeback_pos_record);
  std::memset(h, 0, sizeof(*h));
}

int rvvla_cvr_spmv_f64(const rvvla_cvr* A, double alpha, const double* x, double beta, double* y, void* stream) {
  return cvr_spmv_impl<double, double, double>(A, alpha, x, beta, y, as_stream(stream));
}

int rvvla_cvr_spmv_f32(const rvvla_cvr* A, float alpha, const float* x, float beta, float* y, void* stream) {
  return cvr_spmv_impl<float, float, float>(A, alpha, x, beta, y, as_stream(stream));
}

}  // extern "C"
