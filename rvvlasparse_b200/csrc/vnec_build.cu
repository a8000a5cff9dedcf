// vnec_build.cu — spMtxVNEC structures built on the GPU.  The reference
// builds its partition and IRD on the host in the constructor
// (include/VNEC.h:89-227); the S and D auxiliary arrays its kernels read
// (src/rvv/spmv_mtx_vnec.cpp:78-446) it defines only by use.  Bit for bit the
// oracle's build_vnec:
//
//   partition : merge path of (row ends, nonzero indices) into
//               NUM_THREADS_VNEC pieces of ceil((nnz + m) / NT) items
//               (VNEC.h:89-100, MergePathDivide spmv_mtx_vnec.cpp:42-71);
//   compaction: per piece, its distinct columns ascending (use_x_indices) and
//               each nonzero's rank among them (ecr_indices) (VNEC.h:104-140)
//               — one stable radix sort of (piece, column) over all
//               nonzeros, then unique flags and their scans;
//   groups    : per row part, windows of nLanes consecutive compacted
//               columns (col_start, v_row_ptr, val_align) (VNEC.h:147-177);
//   IRD       : nnz / (groups * nLanes); variant L if m >= 2,000,000, else D
//               if IRD >= 0.437 (fp32) / 0.477 (fp64), else S
//               (VNEC.h:218-226, SpB_mxv_VNEC.h:22-25);
//   S         : pieces of whole rows; per piece the rows shorter than nLanes
//               ordered by length (descending, stable) go in cross-row groups
//               of nLanes rows (padded with value 0 / compacted column 0),
//               the rest — leftover short rows, then long rows in row order —
//               in-row tasks; every row is one task.
#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "devsort.cuh"
#include "rvvla_internal.cuh"
#include "scan.cuh"

namespace rvvla {
namespace {

__device__ void merge_path_dev(int64_t diagonal, const int* a, int64_t a_len, int64_t b_len, int* x, int* y) {
  int64_t lo = max(diagonal - b_len, (int64_t)0), hi = min(diagonal, a_len);
  while (lo < hi) {
    const int64_t piv = (lo + hi) >> 1;
    if ((int64_t)a[piv] <= diagonal - piv - 1) lo = piv + 1;
    else hi = piv;
  }
  *x = (int)min(lo, a_len);
  *y = (int)(diagonal - lo);
}

__global__ void vnec_partition_kernel(int64_t NT, int64_t ipt, int64_t items, const int* __restrict__ Rst, int64_t m,
                                      int64_t nnz, int* __restrict__ tcs, int* __restrict__ tce) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= NT) return;
  const int64_t d0 = min(ipt * t, items), d1 = min(d0 + ipt, items);
  merge_path_dev(d0, Rst + 1, m, nnz, &tcs[2 * t], &tcs[2 * t + 1]);
  merge_path_dev(d1, Rst + 1, m, nnz, &tce[2 * t], &tce[2 * t + 1]);
}

// the last of the n non-decreasing starts that is <= v (stride in ints)
__device__ __forceinline__ int64_t last_le(const int* starts, int64_t n, int stride, int64_t v) {
  int64_t lo = 0, hi = n;  // first index with start > v
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if ((int64_t)starts[mid * stride] <= v) lo = mid + 1;
    else hi = mid;
  }
  return lo - 1;
}

// keys (piece, column) of every nonzero; D pieces split the nonzeros by
// merge path (starts at tcs[2t+1]), S pieces take whole rows (starts at
// tcs[2t], rows -> row_of)
__global__ void vnec_keys_kernel(int64_t nnz, int64_t NT, const int* __restrict__ tcs, const int* __restrict__ Col,
                                 const int* __restrict__ row_of, int by_rows, uint64_t* __restrict__ key,
                                 uint32_t* __restrict__ val) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nnz) return;
  const int64_t t = by_rows ? last_le(tcs, NT, 2, row_of[j]) : last_le(tcs + 1, NT, 2, j);
  key[j] = ((uint64_t)t << 32) | (uint32_t)Col[j];
  val[j] = (uint32_t)j;
}

__global__ void vnec_row_of_kernel(int64_t m, const int* __restrict__ Rst, int* __restrict__ row_of) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= m) return;
  for (int k = Rst[r]; k < Rst[r + 1]; ++k) row_of[k] = (int)r;
}

// The keys are sorted, so a warp's keys fall in a few runs of one piece:
// one atomic per run (the last lane of the run adds the run's distinct keys).
__global__ void vnec_uniq_kernel(int64_t n, const uint64_t* __restrict__ key, int64_t* __restrict__ flag,
                                 int* __restrict__ nec) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const bool valid = p < n;
  const uint64_t k = valid ? key[p] : 0;
  const bool u = valid && (p == 0 || k != key[p - 1]);
  if (valid) flag[p] = u ? 1 : 0;
  const uint32_t piece = (uint32_t)(k >> 32);
  const uint32_t np = __shfl_down_sync(0xffffffffu, piece, 1);
  const bool nvalid = __shfl_down_sync(0xffffffffu, valid, 1);
  const bool last = valid && (lane == 31 || !nvalid || np != piece);
  const unsigned um = __ballot_sync(0xffffffffu, u);
  const unsigned lm = __ballot_sync(0xffffffffu, last);
  if (last) {
    const unsigned below = lm & ((1u << lane) - 1u);
    const int start = below ? 32 - __clz(below) : 0;  // first lane of this run
    const unsigned run = (lane == 31 ? 0xffffffffu : ((2u << lane) - 1u)) & ~((1u << start) - 1u);
    const int cnt = __popc(um & run);
    if (cnt) atomicAdd(nec + piece, cnt);
  }
}

// ranks and the distinct column lists: excl = exclusive scan of the flags
__global__ void vnec_rank_kernel(int64_t n, const uint64_t* __restrict__ key, const uint32_t* __restrict__ val,
                                 const int64_t* __restrict__ flag, const int64_t* __restrict__ excl,
                                 const int* __restrict__ uxp, int* __restrict__ ecr, int* __restrict__ ux) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int64_t u = excl[p] + flag[p] - 1;  // index of this key among the distinct keys
  const int t = (int)(key[p] >> 32);
  ecr[val[p]] = (int)(u - uxp[t]);
  if (flag[p]) ux[u] = (int)(uint32_t)key[p];
}

// groups of one row part (row i of D piece t: nonzeros from max(row start,
// piece start)); fill != 0 also writes col_start / val_align
template <class T>
__global__ void vnec_groups_kernel(int64_t m, int64_t NT, int nL, const int* __restrict__ Rst,
                                   const int* __restrict__ tcs, const int* __restrict__ ecr, const T* __restrict__ Val,
                                   int64_t* __restrict__ gcount, const int* __restrict__ vrp, int* __restrict__ cs,
                                   T* __restrict__ va) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int64_t t = last_le(tcs, NT, 2, i);
  const int ys = t >= 0 ? tcs[2 * t + 1] : 0;
  const int ps = max(Rst[i], ys);
  const int cnt = Rst[i + 1] - ps;
  if (!vrp) {
    int64_t g = 0;
    if (cnt > 0) {
      int c0 = ecr[ps];
      for (int j = 1; j < cnt; ++j)
        if (ecr[ps + j] - c0 >= nL) {
          ++g;
          c0 = ecr[ps + j];
        }
      ++g;
    }
    gcount[i] = g;
    return;
  }
  if (cnt <= 0) return;
  int64_t g = vrp[i];
  int c0 = ecr[ps];
  cs[g] = c0;
  for (int j = 0; j < cnt; ++j) {
    const int e = ecr[ps + j];
    if (e - c0 >= nL) {
      ++g;
      c0 = e;
      cs[g] = c0;
    }
    va[g * nL + (e - c0)] = Val[ps + j];
  }
}

__global__ void vnec_i64_to_i32_kernel(int64_t n, const int64_t* __restrict__ in, int* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (int)in[i];
}

// S: per row, short (< nL) or long; short rows keyed by (piece, length desc)
__global__ void vnec_s_rows_kernel(int64_t m, int64_t NT, int nL, const int* __restrict__ Rst,
                                   const int* __restrict__ tcs, int* __restrict__ spiece, int* __restrict__ nshort,
                                   uint64_t* __restrict__ skey, uint32_t* __restrict__ sval) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= m) return;
  const int64_t t = last_le(tcs, NT, 2, r);
  spiece[r] = (int)t;
  const int len = Rst[r + 1] - Rst[r];
  const bool sh = len < nL;
  // inside a piece: short rows first, by length descending; long rows after
  // them with one key (the stable sort keeps them in row order)
  skey[r] = ((uint64_t)t << 33) | (sh ? (uint64_t)(~(uint32_t)len) : ((uint64_t)1 << 32));
  sval[r] = (uint32_t)r;
  if (sh) atomicAdd(nshort + t, 1);
}

// task of every row: the sorted order (pieces in order; inside a piece short
// rows by length, descending, then long rows in row order); unit size of
// each task: a cross-row group's padded block on its first member (0 on the
// others), an in-row task's length
__global__ void vnec_s_tasks_kernel(int64_t m, int nL, const int* __restrict__ Rst, const uint32_t* __restrict__ sorted,
                                    const int* __restrict__ spiece, const int* __restrict__ tcs,
                                    const int* __restrict__ nshort, int* __restrict__ tasks,
                                    int64_t* __restrict__ unit) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= m) return;
  const uint32_t r = sorted[p];
  const int t = spiece[r];
  const int64_t within = p - tcs[2 * t];  // position among the piece's rows
  const int64_t ngr = nshort[t] / nL;
  const int len = Rst[r + 1] - Rst[r];
  tasks[p] = (int)r;
  if (within < ngr * nL) unit[p] = (within % nL == 0) ? (int64_t)len * nL : 0;
  else unit[p] = len;
}

template <class T>
__global__ void vnec_s_fill_kernel(int64_t m, int nL, const int* __restrict__ Rst, const uint32_t* __restrict__ sorted, const int* __restrict__ spiece,
                                   const int* __restrict__ tcs, const int* __restrict__ nshort,
                                   const int64_t* __restrict__ uoff, const int* __restrict__ ecrS,
                                   const T* __restrict__ Val, int* __restrict__ rb, int* __restrict__ re,
                                   int* __restrict__ rc, T* __restrict__ rv) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= m) return;
  const uint32_t r = sorted[p];
  const int t = spiece[r];
  const int64_t within = p - tcs[2 * t];
  const int64_t ngr = nshort[t] / nL;
  const int k0 = Rst[r], len = Rst[r + 1] - k0;
  if (within < ngr * nL) {
    const int64_t k = within % nL;
    const int64_t lead = p - k;  // the group's first member
    const int64_t base = uoff[lead];
    const int rl = Rst[sorted[lead] + 1] - Rst[sorted[lead]];
    rb[p] = (int)base;
    re[p] = (int)(base + rl);
    for (int c = 0; c < len; ++c) {
      rc[base + (int64_t)c * nL + k] = ecrS[k0 + c];
      rv[base + (int64_t)c * nL + k] = Val[k0 + c];
    }
  } else {
    const int64_t base = uoff[p];
    rb[p] = (int)base;
    re[p] = (int)(base + len);
    for (int c = 0; c < len; ++c) {
      rc[base + c] = ecrS[k0 + c];
      rv[base + c] = Val[k0 + c];
    }
  }
}

__global__ void vnec_s_piece_kernel(int64_t NT, int nL, const int* __restrict__ tcs, int64_t m,
                                    const int* __restrict__ nshort, int* __restrict__ ts, int* __restrict__ te,
                                    int* __restrict__ spv) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= NT) return;
  const int r0 = tcs[2 * t];
  const int r1 = t + 1 < NT ? max(r0, tcs[2 * (t + 1)]) : (int)m;
  ts[t] = r0;
  te[t] = max(r0, r1);
  spv[t] = (nshort[t] / nL) * nL;
}

template <class T>
int dalloc(T** p, int64_t n) {
  RVVLA_CUDA(cudaMalloc(p, (size_t)std::max<int64_t>(n, 1) * sizeof(T)));
  return RVVLA_OK;
}

// sort-unique compaction of the nonzeros by (piece, column): ecr, nec, uxp, ux
int compaction(int64_t nnz, int64_t NT, const int* tcs, const int* Col, const int* row_of, int by_rows, int* ecr,
               int* nec, int* uxp, int** ux, int64_t* nux, cudaStream_t st) {
  RVVLA_CUDA(cudaMemsetAsync(nec, 0, (size_t)std::max<int64_t>(NT, 1) * sizeof(int), st));
  Scratch k1, k2, v1, v2, fl, ex, n64, u64;
  RVVLA_CUDA(k1.alloc((size_t)std::max<int64_t>(nnz, 1) * 8, st));
  RVVLA_CUDA(k2.alloc((size_t)std::max<int64_t>(nnz, 1) * 8, st));
  RVVLA_CUDA(v1.alloc((size_t)std::max<int64_t>(nnz, 1) * 4, st));
  RVVLA_CUDA(v2.alloc((size_t)std::max<int64_t>(nnz, 1) * 4, st));
  RVVLA_CUDA(fl.alloc((size_t)(nnz + 1) * 8, st));
  RVVLA_CUDA(ex.alloc((size_t)(nnz + 1) * 8, st));
  int rc = 0;
  if (nnz > 0) {
    vnec_keys_kernel<<<grid_for(nnz), 256, 0, st>>>(nnz, NT, tcs, Col, row_of, by_rows, k1.as<uint64_t>(),
                                                     v1.as<uint32_t>());
    if ((rc = radix_sort_pairs(k1.as<uint64_t>(), k2.as<uint64_t>(), v1.as<uint32_t>(), v2.as<uint32_t>(), nnz,
                               32 + bits_for((uint64_t)std::max<int64_t>(NT, 1)), st)))
      return rc;
    vnec_uniq_kernel<<<grid_for(nnz), 256, 0, st>>>(nnz, k2.as<uint64_t>(), fl.as<int64_t>(), nec);
    if ((rc = exclusive_scan_i64(fl.as<int64_t>(), ex.as<int64_t>(), nnz, st))) return rc;
  } else {
    RVVLA_CUDA(cudaMemsetAsync(ex.p, 0, 8, st));
  }
  // uxp = exclusive scan of nec
  RVVLA_CUDA(n64.alloc((size_t)(NT + 1) * 8, st));
  RVVLA_CUDA(u64.alloc((size_t)(NT + 1) * 8, st));
  {
    std::vector<int> hn((size_t)NT);
    RVVLA_CUDA(cudaMemcpyAsync(hn.data(), nec, (size_t)NT * sizeof(int), cudaMemcpyDeviceToHost, st));
    RVVLA_CUDA(cudaStreamSynchronize(st));
    std::vector<int> hp((size_t)NT + 1, 0);
    for (int64_t t = 0; t < NT; ++t) hp[(size_t)t + 1] = hp[(size_t)t] + hn[(size_t)t];
    RVVLA_CUDA(cudaMemcpyAsync(uxp, hp.data(), (size_t)(NT + 1) * sizeof(int), cudaMemcpyHostToDevice, st));
    *nux = hp[(size_t)NT];
  }
  if ((rc = dalloc(ux, *nux))) return rc;
  if (nnz > 0)
    vnec_rank_kernel<<<grid_for(nnz), 256, 0, st>>>(nnz, k2.as<uint64_t>(), v2.as<uint32_t>(), fl.as<int64_t>(),
                                                     ex.as<int64_t>(), uxp, ecr, *ux);
  RVVLA_LAUNCHED("vnec compaction kernels");
  RVVLA_CUDA(cudaStreamSynchronize(st));  // the host vectors above leave scope
  return RVVLA_OK;
}

}  // namespace

template <class T>
int vnec_build_gpu(const rvvla_crs* src, int64_t NT, int force, int nL, double thr, rvvla_vnec_owned* out,
                   cudaStream_t st) {
  const int64_t m = src->m, nnz = src->nz, items = nnz + m;
  const int64_t ipt = (items + NT - 1) / NT;
  rvvla_vnec& h = out->h;
  int rc = 0;
  // owned copies of the source CRS
  if ((rc = dalloc(&out->ptr, m + 1)) || (rc = dalloc(&out->indices, nnz)) ||
      (rc = dalloc(reinterpret_cast<T**>(&out->val), nnz)))
    return rc;
  RVVLA_CUDA(cudaMemcpyAsync(out->ptr, src->Rst, (size_t)(m + 1) * 4, cudaMemcpyDeviceToDevice, st));
  if (nnz) {
    RVVLA_CUDA(cudaMemcpyAsync(out->indices, src->Col, (size_t)nnz * 4, cudaMemcpyDeviceToDevice, st));
    RVVLA_CUDA(cudaMemcpyAsync(out->val, src->Val, (size_t)nnz * sizeof(T), cudaMemcpyDeviceToDevice, st));
  }
  const int* Rst = out->ptr;
  const int* Col = out->indices;
  const T* Val = static_cast<const T*>(out->val);
  // partition
  if ((rc = dalloc(&out->thread_coord_start, 2 * NT)) || (rc = dalloc(&out->thread_coord_end, 2 * NT))) return rc;
  vnec_partition_kernel<<<grid_for(NT), 256, 0, st>>>(NT, ipt, items, Rst, m, nnz, out->thread_coord_start,
                                                       out->thread_coord_end);
  RVVLA_LAUNCHED("vnec_partition_kernel");
  const int* tcs = out->thread_coord_start;
  // D compaction (its groups give the IRD for every variant)
  Scratch s_ecr, s_nec, s_uxp, s_gc, s_vrp;
  RVVLA_CUDA(s_ecr.alloc((size_t)std::max<int64_t>(nnz, 1) * 4, st));
  RVVLA_CUDA(s_nec.alloc((size_t)std::max<int64_t>(NT, 1) * 4, st));
  RVVLA_CUDA(s_uxp.alloc((size_t)(NT + 1) * 4, st));
  int* ux_d = nullptr;
  int64_t nux_d = 0;
  if ((rc = compaction(nnz, NT, tcs, Col, nullptr, 0, s_ecr.as<int>(), s_nec.as<int>(), s_uxp.as<int>(), &ux_d,
                       &nux_d, st))) {
    cudaFree(ux_d);
    return rc;
  }
  std::unique_ptr<int, decltype(&cudaFree)> ux_d_hold(ux_d, &cudaFree);
  // group counts per row part, v_row_ptr = their inclusive scan
  RVVLA_CUDA(s_gc.alloc((size_t)(m + 1) * 8, st));
  RVVLA_CUDA(s_vrp.alloc((size_t)(m + 1) * 8, st));
  int64_t ngroups = 0;
  if (m > 0) {
    vnec_groups_kernel<T><<<grid_for(m), 256, 0, st>>>(m, NT, nL, Rst, tcs, s_ecr.as<int>(), Val,
                                                        s_gc.as<int64_t>(), nullptr, nullptr, nullptr);
    if ((rc = exclusive_scan_i64(s_gc.as<int64_t>(), s_vrp.as<int64_t>(), m, st))) return rc;
    RVVLA_CUDA(cudaMemcpyAsync(&ngroups, s_vrp.as<int64_t>() + m, 8, cudaMemcpyDeviceToHost, st));
  }
  RVVLA_LAUNCHED("vnec_groups_kernel");
  std::vector<int> nec_h((size_t)NT);
  RVVLA_CUDA(cudaMemcpyAsync(nec_h.data(), s_nec.p, (size_t)NT * 4, cudaMemcpyDeviceToHost, st));
  RVVLA_CUDA(cudaStreamSynchronize(st));
  const double ird = ngroups > 0 ? (double)nnz / ((double)ngroups * nL) : 0.0;
  h.IRD_mat = (float)ird;
  int variant;
  if (force >= 0) variant = force;
  else if (m < 2000000) variant = (h.IRD_mat >= (float)thr) ? 0 : 1;
  else variant = 2;
  h.vnec_t = variant;
  int max_nec = 0;
  for (int v : nec_h) max_nec = std::max(max_nec, v);
  if (variant == 0) {
    // the D structures: the compaction above plus the groups' columns and values
    if ((rc = dalloc(&out->ecr_indices, nnz)) || (rc = dalloc(&out->NEC_NUM, NT)) ||
        (rc = dalloc(&out->use_x_ptr, NT + 1)) || (rc = dalloc(&out->v_row_ptr, m + 1)) ||
        (rc = dalloc(&out->col_start, ngroups)) || (rc = dalloc(reinterpret_cast<T**>(&out->val_align), ngroups * nL)))
      return rc;
    RVVLA_CUDA(cudaMemcpyAsync(out->ecr_indices, s_ecr.p, (size_t)std::max<int64_t>(nnz, 1) * 4,
                               cudaMemcpyDeviceToDevice, st));
    RVVLA_CUDA(cudaMemcpyAsync(out->NEC_NUM, s_nec.p, (size_t)NT * 4, cudaMemcpyDeviceToDevice, st));
    RVVLA_CUDA(cudaMemcpyAsync(out->use_x_ptr, s_uxp.p, (size_t)(NT + 1) * 4, cudaMemcpyDeviceToDevice, st));
    out->use_x_indices = ux_d_hold.release();
    // v_row_ptr[i + 1] = groups through row i
    RVVLA_CUDA(cudaMemsetAsync(out->v_row_ptr, 0, 4, st));
    vnec_i64_to_i32_kernel<<<grid_for(m), 256, 0, st>>>(m, s_vrp.as<int64_t>() + 1, out->v_row_ptr + 1);
    RVVLA_CUDA(cudaMemsetAsync(out->val_align, 0, (size_t)std::max<int64_t>(ngroups * nL, 1) * sizeof(T), st));
    {
      Scratch s_v32;
      RVVLA_CUDA(s_v32.alloc((size_t)(m + 1) * 4, st));
      vnec_i64_to_i32_kernel<<<grid_for(m + 1), 256, 0, st>>>(m + 1, s_vrp.as<int64_t>(), s_v32.as<int>());
      if (m > 0)
        vnec_groups_kernel<T><<<grid_for(m), 256, 0, st>>>(m, NT, nL, Rst, tcs, out->ecr_indices, Val, nullptr,
                                                            s_v32.as<int>(), out->col_start,
                                                            static_cast<T*>(out->val_align));
      RVVLA_LAUNCHED("vnec D fill kernels");
      RVVLA_CUDA(cudaStreamSynchronize(st));
    }
    h.ngroups = ngroups;
  } else if (variant == 1) {
    // the S structures: compaction over whole-row pieces, tasks, reordered rows
    Scratch s_rowof, s_sp, s_ns, s_sk, s_sk2, s_sv, s_sorted, s_unit, s_uoff, s_ecrS;
    RVVLA_CUDA(s_rowof.alloc((size_t)std::max<int64_t>(nnz, 1) * 4, st));
    if (m > 0) vnec_row_of_kernel<<<grid_for(m), 256, 0, st>>>(m, Rst, s_rowof.as<int>());
    if ((rc = dalloc(&out->NEC_NUM, NT)) || (rc = dalloc(&out->use_x_ptr, NT + 1))) return rc;
    RVVLA_CUDA(s_ecrS.alloc((size_t)std::max<int64_t>(nnz, 1) * 4, st));
    int64_t nux_s = 0;
    if ((rc = compaction(nnz, NT, tcs, Col, s_rowof.as<int>(), 1, s_ecrS.as<int>(), out->NEC_NUM, out->use_x_ptr,
                         &out->use_x_indices, &nux_s, st)))
      return rc;
    RVVLA_CUDA(s_sp.alloc((size_t)std::max<int64_t>(m, 1) * 4, st));
    RVVLA_CUDA(s_ns.alloc((size_t)std::max<int64_t>(NT, 1) * 4, st));
    RVVLA_CUDA(cudaMemsetAsync(s_ns.p, 0, (size_t)std::max<int64_t>(NT, 1) * 4, st));
    RVVLA_CUDA(s_sk.alloc((size_t)std::max<int64_t>(m, 1) * 8, st));
    RVVLA_CUDA(s_sk2.alloc((size_t)std::max<int64_t>(m, 1) * 8, st));
    RVVLA_CUDA(s_sv.alloc((size_t)std::max<int64_t>(m, 1) * 4, st));
    RVVLA_CUDA(s_sorted.alloc((size_t)std::max<int64_t>(m, 1) * 4, st));
    if (m > 0) {
      vnec_s_rows_kernel<<<grid_for(m), 256, 0, st>>>(m, NT, nL, Rst, tcs, s_sp.as<int>(), s_ns.as<int>(),
                                                      s_sk.as<uint64_t>(), s_sv.as<uint32_t>());
      if ((rc = radix_sort_pairs(s_sk.as<uint64_t>(), s_sk2.as<uint64_t>(), s_sv.as<uint32_t>(),
                                 s_sorted.as<uint32_t>(), m, 33 + bits_for((uint64_t)std::max<int64_t>(NT, 1)), st)))
        return rc;
    }
    if ((rc = dalloc(&out->tasks, m)) || (rc = dalloc(&out->task_start, NT)) || (rc = dalloc(&out->task_end, NT)) ||
        (rc = dalloc(&out->spvv_len, NT)) || (rc = dalloc(&out->row_begin, m)) || (rc = dalloc(&out->row_end, m)))
      return rc;
    RVVLA_CUDA(s_unit.alloc((size_t)(m + 1) * 8, st));
    RVVLA_CUDA(s_uoff.alloc((size_t)(m + 1) * 8, st));
    int64_t nreorder = 0;
    if (m > 0) {
      vnec_s_tasks_kernel<<<grid_for(m), 256, 0, st>>>(m, nL, Rst, s_sorted.as<uint32_t>(), s_sp.as<int>(), tcs,
                                                       s_ns.as<int>(), out->tasks, s_unit.as<int64_t>());
      if ((rc = exclusive_scan_i64(s_unit.as<int64_t>(), s_uoff.as<int64_t>(), m, st))) return rc;
      RVVLA_CUDA(cudaMemcpyAsync(&nreorder, s_uoff.as<int64_t>() + m, 8, cudaMemcpyDeviceToHost, st));
      RVVLA_CUDA(cudaStreamSynchronize(st));
    }
    if ((rc = dalloc(&out->reorder_col, nreorder)) || (rc = dalloc(reinterpret_cast<T**>(&out->reorder_nnz), nreorder)))
      return rc;
    RVVLA_CUDA(cudaMemsetAsync(out->reorder_col, 0, (size_t)std::max<int64_t>(nreorder, 1) * 4, st));
    RVVLA_CUDA(cudaMemsetAsync(out->reorder_nnz, 0, (size_t)std::max<int64_t>(nreorder, 1) * sizeof(T), st));
    if (m > 0)
      vnec_s_fill_kernel<T><<<grid_for(m), 256, 0, st>>>(m, nL, Rst, s_sorted.as<uint32_t>(), s_sp.as<int>(),
                                                          tcs, s_ns.as<int>(), s_uoff.as<int64_t>(), s_ecrS.as<int>(),
                                                          Val, out->row_begin, out->row_end, out->reorder_col,
                                                          static_cast<T*>(out->reorder_nnz));
    vnec_s_piece_kernel<<<grid_for(NT), 256, 0, st>>>(NT, nL, tcs, m, s_ns.as<int>(), out->task_start, out->task_end,
                                                      out->spvv_len);
    RVVLA_LAUNCHED("vnec S kernels");
    std::vector<int> ns_h((size_t)NT);
    RVVLA_CUDA(cudaMemcpyAsync(ns_h.data(), out->NEC_NUM, (size_t)NT * 4, cudaMemcpyDeviceToHost, st));
    RVVLA_CUDA(cudaStreamSynchronize(st));
    max_nec = 0;
    for (int v : ns_h) max_nec = std::max(max_nec, v);
    h.ntasks = m;
    h.nreorder = nreorder;
  }
  h.max_nec = max_nec;
  RVVLA_CUDA(cudaStreamSynchronize(st));
  return RVVLA_OK;
}

template int vnec_build_gpu<double>(const rvvla_crs*, int64_t, int, int, double, rvvla_vnec_owned*, cudaStream_t);
template int vnec_build_gpu<float>(const rvvla_crs*, int64_t, int, int, double, rvvla_vnec_owned*, cudaStream_t);

}  // namespace rvvla
